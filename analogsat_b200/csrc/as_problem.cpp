// Host-side CNF storage, DIMACS IO and device packing (see as_problem.h).
#include "as_problem.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>

namespace asb {

void HostProblem::add_clauses(const int32_t* literals, const int32_t* lengths, int count) {
    int offset = 0;
    for (int j = 0; j < count; j++) {
        const int len = lengths[j];
        const int st = (int)storage.size();
        int kept = 0, n_new = n;
        for (int i = 0; i < len; i++) {
            const int lit = literals[offset++];
            if (lit == 0) continue;
            storage.push_back(lit);
            n_new = std::max(n_new, std::abs(lit));
            kept++;
        }
        if (kept == 0) continue;  // empty clauses are dropped (SatProblem.cpp:52)
        start.push_back(st);
        length.push_back(kept);
        k = std::max(k, kept);
        n = n_new;
        m++;
    }
}

// Same acceptance rules as CnfReader::Read: lines before the "p cnf N M" header are
// skipped, a header with N == 0 or M == 0 is an empty problem, then exactly M
// zero-terminated clauses must follow.
bool read_cnf(const char* path, HostProblem& p, std::string& msg) {
    FILE* f = std::fopen(path, "r");
    if (!f) { msg = "file open failed"; return false; }
    int n = -1, m = -1;
    char line[1024];
    while (!std::feof(f)) {
        int c = std::fgetc(f);
        if (c == EOF) break;
        if (c == 'p') {
            if (std::fscanf(f, " cnf %d %d", &n, &m) == 2) break;
            msg = "expected: p cnf <variables> <clauses>";
            std::fclose(f);
            return false;
        }
        if (c != '\n' && !std::fgets(line, sizeof(line), f)) break;
    }
    if (n < 0 || m < 0) { msg = "could not find a SAT declaration"; std::fclose(f); return false; }
    p = HostProblem();
    if (n == 0 || m == 0) { msg = "empty problem"; std::fclose(f); return true; }
    std::vector<int32_t> lits, lens;
    lits.reserve((size_t)m * 3);
    lens.reserve(m);
    int read = 0;
    while (read < m) {
        int len = 0;
        while (true) {
            int lit;
            if (std::fscanf(f, "%d", &lit) != 1) {
                msg = "expected more literals in file";
                std::fclose(f);
                return false;
            }
            if (lit == 0) break;
            lits.push_back(lit);
            len++;
        }
        lens.push_back(len);
        read++;
    }
    std::fclose(f);
    p.add_clauses(lits.data(), lens.data(), (int)lens.size());
    msg = "read ok";
    return true;
}

bool write_cnf(const char* path, const HostProblem& p) {
    FILE* f = std::fopen(path, "w");
    if (!f) return false;
    std::fprintf(f, "p cnf %d %d\n", p.n, p.m);
    for (int j = 0; j < p.m; j++) {
        for (int i = 0; i < p.length[j]; i++) std::fprintf(f, "%d ", p.storage[p.start[j] + i]);
        std::fprintf(f, "0\n");
    }
    std::fclose(f);
    return true;
}

PackedProblem pack(const HostProblem& p) {
    PackedProblem q;
    q.n = p.n;
    q.m = p.m;
    q.k = p.k;
    q.mp = std::max(32, (p.m + 31) / 32 * 32);
    q.nslices = (p.n + 31) / 32;

    // degree of every public variable and its incidences in (clause, slot) order
    std::vector<int32_t> degree(p.n, 0);
    for (int j = 0; j < p.m; j++)
        for (int i = 0; i < p.length[j]; i++) degree[std::abs(p.storage[p.start[j] + i]) - 1]++;
    q.max_degree = 0;
    for (int v = 0; v < p.n; v++) q.max_degree = std::max(q.max_degree, degree[v]);

    // internal order: decreasing degree, ties by public index
    q.perm.resize(p.n);
    for (int v = 0; v < p.n; v++) q.perm[v] = v;
    std::stable_sort(q.perm.begin(), q.perm.end(),
                     [&](int a, int b) { return degree[a] > degree[b]; });
    q.iperm.resize(p.n);
    for (int v = 0; v < p.n; v++) q.iperm[q.perm[v]] = v;

    // SELL-32 rows: slice g is as wide as its largest degree
    q.srow.assign(q.nslices + 1, 0);
    for (int g = 0; g < q.nslices; g++) {
        int w = 0;
        for (int l = 0; l < 32 && g * 32 + l < p.n; l++) w = std::max(w, degree[q.perm[g * 32 + l]]);
        q.srow[g + 1] = q.srow[g] + w;
    }
    q.nslots = q.srow[q.nslices] * 32;
    q.compact = p.n < 32768 && q.nslots <= 65535;

    const uint32_t pad = ((uint32_t)std::min(p.n, 32767) << 16) | (uint32_t)std::min(q.nslots, 65535);
    q.lit.assign((size_t)q.k * q.mp, pad);
    std::vector<int32_t> rank(p.n, 0);  // next row of each internal variable
    for (int j = 0; j < p.m; j++) {
        for (int i = 0; i < p.length[j]; i++) {
            const int lit = p.storage[p.start[j] + i];
            const int v = q.iperm[std::abs(lit) - 1];
            const int slot = (q.srow[v >> 5] + rank[v]++) * 32 + (v & 31);
            if (q.compact)
                q.lit[(size_t)i * q.mp + j] =
                    (lit < 0 ? 0x80000000u : 0u) | ((uint32_t)v << 16) | (uint32_t)slot;
        }
    }
    return q;
}

}  // namespace asb
