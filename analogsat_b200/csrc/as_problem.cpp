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

namespace {

// Greedy bank-aware grouping of clauses into warps of 32 (see as_problem.h): take
// clauses in a shuffled order, put a clause into the open group when its literal
// banks (optionally after reordering its literals) are all still free in their
// slots; when no candidate within a search window fits, complete the group with the
// least-conflicting candidates.  Deterministic (fixed seed).
void schedule_clauses(const HostProblem& p, PackedProblem& q, bool permute, bool pairs,
                      std::vector<std::vector<int8_t>>& order) {
    const int m = p.m, k = p.k;
    order.assign(m, {});
    q.cperm.resize(m);
    q.icperm.resize(m);
    // 32-bit layouts: bank = internal variable mod 32, one set of 32 lanes;
    // pair layout: bank pair = internal variable mod 16, per 16-lane half
    const int lanes = pairs ? 16 : 32;
    std::vector<int32_t> bank(p.storage.size());
    for (size_t i = 0; i < p.storage.size(); i++) bank[i] = q.iperm[std::abs(p.storage[i]) - 1] & (lanes - 1);
    // candidate literal orders per clause length (all permutations for k <= 4)
    auto perms_for = [&](int len) {
        std::vector<std::vector<int8_t>> ps;
        std::vector<int8_t> id(len);
        for (int i = 0; i < len; i++) id[i] = (int8_t)i;
        if (!permute || len > 4) { ps.push_back(id); return ps; }
        do ps.push_back(id); while (std::next_permutation(id.begin(), id.end()));
        return ps;
    };
    std::vector<std::vector<std::vector<int8_t>>> perms(k + 1);
    for (int len = 1; len <= k; len++) perms[len] = perms_for(len);

    std::vector<int32_t> rem(m);
    for (int j = 0; j < m; j++) rem[j] = j;
    uint64_t rng = 0x9E3779B97F4A7C15ull;
    for (int j = m - 1; j > 0; j--) {  // Fisher-Yates with an xorshift generator
        rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17;
        std::swap(rem[j], rem[rng % (uint64_t)(j + 1)]);
    }
    const int kw = std::min(k, 16);
    // candidates tried per lane (first fit), and per lane of the least-conflict completion
    const size_t kScanWindow = pairs ? 4096 : 1024;
    const int kFillWindow = pairs ? 1024 : 256;
    int out = 0;
    long waves = 0;
    std::vector<uint32_t> used(kw);
    uint32_t used_clause = 0;  // pair layout: public clause index mod 32 across the warp
    std::vector<int32_t> keep;
    keep.reserve(m);
    while (!rem.empty()) {
        std::fill(used.begin(), used.end(), 0u);
        used_clause = 0;
        int filled = 0;
        keep.clear();
        size_t scanned = 0;
        auto cost = [&](int j, const std::vector<int8_t>& ord) {
            int c = pairs ? (int)((used_clause >> (j & 31)) & 1u) : 0;
            for (int qq = 0; qq < (int)ord.size() && qq < kw; qq++)
                c += (used[qq] >> bank[p.start[j] + ord[qq]]) & 1u;
            return c;
        };
        auto take = [&](int j, const std::vector<int8_t>& ord) {
            for (int qq = 0; qq < (int)ord.size() && qq < kw; qq++)
                used[qq] |= 1u << bank[p.start[j] + ord[qq]];
            used_clause |= 1u << (j & 31);
            order[out] = ord;
            q.cperm[out] = j;
            out++;
            filled++;
            if (filled == lanes && lanes < 32) std::fill(used.begin(), used.end(), 0u);  // second half
        };
        size_t i = 0;
        for (; i < rem.size() && filled < 32; i++) {
            const int j = rem[i];
            bool placed = false;
            if (scanned < kScanWindow) {
                scanned++;
                for (const auto& ord : perms[p.length[j]])
                    if (cost(j, ord) == 0) { take(j, ord); placed = true; break; }
            }
            if (!placed) keep.push_back(j);
        }
        for (; i < rem.size(); i++) keep.push_back(rem[i]);
        while (filled < 32 && !keep.empty()) {
            int best = 0, bc = 1 << 30;
            const std::vector<int8_t>* bo = nullptr;
            for (int c = 0; c < (int)keep.size() && c < kFillWindow; c++) {
                for (const auto& ord : perms[p.length[keep[c]]]) {
                    const int cc = cost(keep[c], ord);
                    if (cc < bc) { bc = cc; best = c; bo = &ord; }
                }
                if (bc == 0) break;
            }
            const int j = keep[best];
            const std::vector<int8_t> ord = *bo;
            std::swap(keep[best], keep.back());
            keep.pop_back();
            take(j, ord);
        }
        rem.swap(keep);
    }
    for (int mi = 0; mi < m; mi++) q.icperm[q.cperm[mi]] = mi;
    // wavefront count of one gather pass (per bank group of `lanes` clauses), for diagnostics
    for (int g = 0; g < m; g += lanes) {
        for (int qq = 0; qq < kw; qq++) {
            int cnt[32] = {0}, mx = 0;
            for (int mi = g; mi < std::min(m, g + lanes); mi++) {
                const int j = q.cperm[mi];
                if (qq < p.length[j]) mx = std::max(mx, ++cnt[bank[p.start[j] + order[mi][qq]]]);
            }
            waves += std::max(mx, 1);
        }
    }
    q.bank_wavefronts = waves;
}

}  // namespace

PackedProblem pack(const HostProblem& p, int mode) {
    const bool permute_literals = mode != kPackReference;
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

    // slot of every literal (rank in its variable's public-ordered incidence list)
    std::vector<int32_t> slot_of(p.storage.size(), 0);
    {
        std::vector<int32_t> rank(p.n, 0);
        for (int j = 0; j < p.m; j++)
            for (int i = 0; i < p.length[j]; i++) {
                const int v = q.iperm[std::abs(p.storage[p.start[j] + i]) - 1];
                slot_of[p.start[j] + i] = (q.srow[v >> 5] + rank[v]++) * 32 + (v & 31);
            }
    }

    // literal order inside each internal clause (indices into the public clause)
    std::vector<std::vector<int8_t>> order;
    if (q.compact) {
        schedule_clauses(p, q, permute_literals, mode == kPackF32Pair, order);
    } else {  // the streamed kernels read no shared-memory banks this way: keep the order
        q.cperm.resize(p.m);
        q.icperm.resize(p.m);
        order.assign(p.m, {});
        for (int j = 0; j < p.m; j++) {
            q.cperm[j] = q.icperm[j] = j;
            for (int i = 0; i < p.length[j]; i++) order[j].push_back((int8_t)i);
        }
    }

    const size_t nw = (size_t)q.k * q.mp;
    q.litw.assign(nw, (uint32_t)p.n);
    q.slotw.assign(nw, (uint32_t)q.nslots);
    if (q.compact) q.lit.assign(nw, ((uint32_t)p.n << 16) | (uint32_t)q.nslots);
    for (int mi = 0; mi < p.m; mi++) {
        const int j = q.cperm[mi];
        for (int qq = 0; qq < p.length[j]; qq++) {
            const int li = p.start[j] + order[mi][qq];
            const int lit = p.storage[li];
            const uint32_t v = (uint32_t)q.iperm[std::abs(lit) - 1];
            const uint32_t neg = lit < 0 ? 0x80000000u : 0u;
            const size_t idx = (size_t)qq * q.mp + mi;
            q.litw[idx] = neg | v;
            q.slotw[idx] = (uint32_t)slot_of[li];
            if (q.compact) q.lit[idx] = neg | (v << 16) | (uint32_t)slot_of[li];
        }
    }
    return q;
}

}  // namespace asb
