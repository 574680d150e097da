// Host-side CNF storage, DIMACS IO and device packing (see as_problem.h).
#include "as_problem.h"

#include <functional>
#include <unordered_map>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace asb {

void HostProblem::add_clauses(const int32_t* literals, const int32_t* lengths, int count) {
    size_t total = 0;
    for (int j = 0; j < count; j++) total += (size_t)std::max(lengths[j], 0);
    storage.reserve(storage.size() + total);
    start.reserve(start.size() + count);
    length.reserve(length.size() + count);
    size_t offset = 0;
    int n_max = n, k_max = k, kept_clauses = 0;
    for (int j = 0; j < count; j++) {
        const int len = lengths[j];
        const int st = (int)storage.size();
        int kept = 0;
        for (int i = 0; i < len; i++) {
            const int lit = literals[offset++];
            if (lit == 0) continue;
            storage.push_back(lit);
            n_max = std::max(n_max, std::abs(lit));
            kept++;
        }
        if (kept == 0) continue;  // empty clauses are dropped (SatProblem.cpp:52)
        start.push_back(st);
        length.push_back(kept);
        k_max = std::max(k_max, kept);
        kept_clauses++;
    }
    n = n_max;
    k = k_max;
    m += kept_clauses;
}

void HostProblem::set_clauses(std::vector<int32_t>&& literals, const std::vector<int32_t>& lengths) {
    *this = HostProblem();
    storage = std::move(literals);
    start.reserve(lengths.size());
    length.reserve(lengths.size());
    int32_t off = 0;
    for (const int32_t len : lengths) {
        if (len > 0) {  // empty clauses are dropped (SatProblem.cpp:84)
            start.push_back(off);
            length.push_back(len);
            k = std::max(k, (int)len);
            m++;
        }
        off += len;
    }
    int nmax = 0;
    for (const int32_t v : storage) nmax = std::max(nmax, v < 0 ? -v : v);
    n = nmax;
}

// Lines before the declaration are skipped whole (CnfReader.cpp:61-82); an empty line
// is skipped on its own rather than taking the next line with it.
bool read_cnf_header(std::FILE* f, int& n, int& m, std::string& msg) {
    n = -1;
    m = -1;
    char line[1024];
    while (!std::feof(f)) {
        int c = std::fgetc(f);
        if (c == EOF) break;
        if (c == 'p') {
            if (std::fscanf(f, " cnf %d %d", &n, &m) == 2) break;
            msg = "expected: p cnf <variables> <clauses>";
            return false;
        }
        if (c != '\n' && !std::fgets(line, sizeof(line), f)) break;
    }
    if (n < 0 || m < 0) { msg = "could not find a SAT declaration"; return false; }
    return true;
}

// Same acceptance rules as CnfReader::Read: lines before the "p cnf N M" header are
// skipped, a header with N == 0 or M == 0 is an empty problem, then exactly M
// zero-terminated clauses must follow.  Literals are read as long and must lie within
// +-(2^31 - 1): the reference's "%d" leaves larger values undefined.
bool read_cnf(const char* path, HostProblem& p, std::string& msg) {
    FILE* f = std::fopen(path, "r");
    if (!f) { msg = "file open failed"; return false; }
    int n = -1, m = -1;
    if (!read_cnf_header(f, n, m, msg)) { std::fclose(f); return false; }
    p = HostProblem();
    if (n == 0 || m == 0) { msg = "empty problem"; std::fclose(f); return true; }
    // the rest of the file in one read, then the clause body by fscanf's rules
    std::vector<char> body;
    char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) body.insert(body.end(), chunk, chunk + got);
    std::fclose(f);
    std::vector<int32_t> lits, lens;
    if (!parse_cnf_body_host(body.data(), body.size(), m, lits, lens, msg)) return false;
    p.set_clauses(std::move(lits), lens);
    msg = "read ok";
    return true;
}

// CnfReader.cpp:100-127 reads the body with fscanf("%d") until M zeros are read:
// skip white space (C locale), an optional sign, at least one digit, greedily.  The
// same reads here over the bytes in memory, with "%ld"'s range checked instead of
// "%d"'s undefined overflow.
bool parse_cnf_body_host(const char* b, size_t len, long long m, std::vector<int32_t>& lits,
                         std::vector<int32_t>& lens, std::string& msg) {
    auto space = [](unsigned char c) { return c == ' ' || (c >= '\t' && c <= '\r'); };
    auto digit = [](unsigned char c) { return c >= '0' && c <= '9'; };
    lits.clear();
    lens.clear();
    lits.reserve(std::min<size_t>(len / 2 + 1, (size_t)m * 3));
    lens.reserve(std::min<size_t>(len / 2 + 1, (size_t)m));
    size_t i = 0;
    int cur = 0;
    long long zeros = 0;
    while (zeros < m) {
        while (i < len && space((unsigned char)b[i])) i++;
        bool neg = false;
        if (i < len && (b[i] == '+' || b[i] == '-')) {
            neg = b[i] == '-';
            i++;
        }
        if (i >= len || !digit((unsigned char)b[i])) {
            msg = "expected more literals in file";
            return false;
        }
        long long v = 0;
        bool range = false;
        for (; i < len && digit((unsigned char)b[i]); i++)
            if (!range) {
                v = v * 10 + (b[i] - '0');
                range = v > 2147483647LL;
            }
        if (range) {
            msg = "literal out of range";
            return false;
        }
        if (v == 0) {
            lens.push_back(cur);
            cur = 0;
            zeros++;
        } else {
            lits.push_back((int32_t)(neg ? -v : v));
            cur++;
        }
    }
    return true;
}

// The text of CnfWriter::Write ("p cnf N M", then per clause "%d " per literal and
// "0"), formatted into a buffer instead of one fprintf per literal.
bool write_cnf(const char* path, const HostProblem& p) {
    FILE* f = std::fopen(path, "w");
    if (!f) return false;
    std::string out;
    out.reserve((size_t)p.storage.size() * 8 + (size_t)p.m * 2 + 64);
    char buf[32];
    out += "p cnf " + std::to_string(p.n) + " " + std::to_string(p.m) + "\n";
    auto put_int = [&](int v) {
        char* e = buf + sizeof buf;
        char* q = e;
        unsigned u = v < 0 ? 0u - (unsigned)v : (unsigned)v;
        do { *--q = (char)('0' + u % 10); u /= 10; } while (u);
        if (v < 0) *--q = '-';
        out.append(q, e);
    };
    for (int j = 0; j < p.m; j++) {
        for (int i = 0; i < p.length[j]; i++) {
            put_int(p.storage[p.start[j] + i]);
            out += ' ';
        }
        out += "0\n";
    }
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return std::fclose(f) == 0 && ok;
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
    // candidates tried by first fit per bank group, and per lane of the least-conflict
    // completion
    const size_t kScanWindow = pairs ? 8192 : 1024;
    const int kFillWindow = pairs ? 1024 : 256;
    int out = 0;
    long waves = 0;
    std::vector<uint32_t> used(kw);
    uint32_t used_clause = 0;  // pair layout: public clause index mod 32 across the warp
    std::vector<int32_t> keep;
    keep.reserve(m);
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
    };
    while (!rem.empty()) {  // one warp of 32 clauses: 32 / lanes bank groups
        used_clause = 0;
        for (int h = 0; h < 32 / lanes && !rem.empty(); h++) {
            std::fill(used.begin(), used.end(), 0u);
            int filled = 0;
            keep.clear();
            size_t scanned = 0, i = 0;
            for (; i < rem.size() && filled < lanes; i++) {
                const int j = rem[i];
                bool placed = false;
                if (scanned < kScanWindow) {
                    scanned++;
                    for (const auto& ord : perms[p.length[j]])
                        if (cost(j, ord) == 0) { take(j, ord); filled++; placed = true; break; }
                }
                if (!placed) keep.push_back(j);
            }
            for (; i < rem.size(); i++) keep.push_back(rem[i]);
            while (filled < lanes && !keep.empty()) {
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
                filled++;
            }
            rem.swap(keep);
        }
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

// Literal slots of one bank group: a bipartite edge colouring (colours = literal
// slots) of the graph lanes x banks whose edges are the group's literals.  A
// bipartite multigraph of maximum degree k is k-edge-colourable (Koenig), so when no
// bank carries more than k literals every slot sees every bank at most once.  The
// literals a bank carries beyond k are set aside first; the rest is coloured one
// edge at a time (when the two ends have different free colours a / b, the a/b
// alternating path from the bank end is recoloured first), and the set-aside edges
// then take colours still free at their clause (a clause has at most k literals, so
// there are enough).
void colour_group(const std::vector<std::vector<int32_t>>& banks, int nbanks, int k,
                  std::vector<std::vector<int8_t>>& slots) {
    const int L = (int)banks.size();
    std::vector<int> eu, ev, ei, ec;
    std::vector<int> deg(nbanks, 0);
    std::vector<char> aside;
    for (int u = 0; u < L; u++)
        for (int i = 0; i < (int)banks[u].size(); i++) {
            eu.push_back(u);
            ev.push_back(banks[u][i]);
            ei.push_back(i);
            ec.push_back(-1);
            aside.push_back(++deg[banks[u][i]] > k);
        }
    const int E = (int)eu.size();
    std::vector<int> colL((size_t)L * k, -1), colR((size_t)nbanks * k, -1);
    for (int e = 0; e < E; e++) {
        if (aside[e]) continue;
        const int u = eu[e], v = ev[e];
        int a = -1, b = -1;
        for (int c = 0; c < k && a < 0; c++)
            if (colL[(size_t)u * k + c] < 0) a = c;
        for (int c = 0; c < k && b < 0; c++)
            if (colR[(size_t)v * k + c] < 0) b = c;
        if (colR[(size_t)v * k + a] >= 0) {
            // alternating a/b path from v: v -a- u1 -b- v2 -a- u2 ... (never reaches u,
            // which has a free); swapping a and b along it frees a at v
            std::vector<int> path;
            int x = v, side = 1, c = a;
            while (true) {
                const int f = side ? colR[(size_t)x * k + c] : colL[(size_t)x * k + c];
                if (f < 0) break;
                path.push_back(f);
                x = side ? eu[f] : ev[f];
                side ^= 1;
                c = c == a ? b : a;
            }
            for (int f : path) {
                colL[(size_t)eu[f] * k + ec[f]] = -1;
                colR[(size_t)ev[f] * k + ec[f]] = -1;
            }
            for (int f : path) {
                ec[f] = ec[f] == a ? b : a;
                colL[(size_t)eu[f] * k + ec[f]] = f;
                colR[(size_t)ev[f] * k + ec[f]] = f;
            }
        }
        ec[e] = a;
        colL[(size_t)u * k + a] = e;
        colR[(size_t)v * k + a] = e;
    }
    for (int e = 0; e < E; e++) {
        if (!aside[e]) continue;
        const int u = eu[e];
        for (int c = 0; c < k; c++)
            if (colL[(size_t)u * k + c] < 0) {
                ec[e] = c;
                colL[(size_t)u * k + c] = e;
                break;
            }
    }
    slots.assign(L, std::vector<int8_t>(k, -1));
    for (int e = 0; e < E; e++) slots[eu[e]][ec[e]] = (int8_t)ei[e];
}

// Local repair of a grouping: while a group holds more than k literals in some bank
// (or, for the pair layout, its warp repeats a public clause index mod 32), swap one
// of its clauses that touches the excess with a clause of another group when that
// lowers the excess of the groups and warps involved.  Candidates are scanned from a
// rotating start (512 candidates per clause), two passes.
void repair_groups(const HostProblem& p, const std::vector<int32_t>& bank, int lanes, int k, bool pairs,
                   std::vector<std::vector<int32_t>>& groups) {
    const int G = (int)groups.size();
    if (G < 2) return;
    std::vector<int32_t> cnt((size_t)G * 32, 0), cj((size_t)G * 32, 0);
    const int kClauseClash = 3;  // as in schedule_balanced
    auto warp = [&](int g) { return pairs ? g / 2 : g; };
    for (int g = 0; g < G; g++)
        for (int j : groups[g]) {
            for (int i = 0; i < p.length[j]; i++) cnt[(size_t)g * 32 + bank[p.start[j] + i]]++;
            cj[(size_t)warp(g) * 32 + (j & 31)]++;
        }
    auto bad = [&](int g) {
        for (int b = 0; b < lanes; b++)
            if (cnt[(size_t)g * 32 + b] > k) return true;
        if (pairs)
            for (int r = 0; r < 32; r++)
                if (cj[(size_t)warp(g) * 32 + r] > 1) return true;
        return false;
    };
    // does clause c of group g touch its excess?
    auto involved = [&](int c, int g) {
        for (int i = 0; i < p.length[c]; i++)
            if (cnt[(size_t)g * 32 + bank[p.start[c] + i]] > k) return true;
        return pairs && cj[(size_t)warp(g) * 32 + (c & 31)] > 1;
    };
    // change of excess when c (in a) and d (in b) trade places
    auto delta = [&](int c, int a, int d, int b) {
        int e = 0;
        int bx[32], nb = 0;
        int dA[32] = {0};
        for (int i = 0; i < p.length[c]; i++) { const int x = bank[p.start[c] + i]; if (!dA[x]++) bx[nb++] = x; }
        for (int i = 0; i < p.length[d]; i++) { const int x = bank[p.start[d] + i]; if (!dA[x]--) bx[nb++] = x; }
        // dA[x] = (# of x in c) - (# of x in d): a loses dA, b gains dA
        for (int t = 0; t < nb; t++) {
            const int x = bx[t], dd = dA[x];
            if (!dd) continue;
            const int ca = cnt[(size_t)a * 32 + x], cb = cnt[(size_t)b * 32 + x];
            e += std::max(0, ca - dd - k) - std::max(0, ca - k);
            e += std::max(0, cb + dd - k) - std::max(0, cb - k);
        }
        if (pairs && warp(a) != warp(b) && ((c ^ d) & 31)) {
            const int rc = c & 31, rd = d & 31;
            const size_t wa = (size_t)warp(a) * 32, wb = (size_t)warp(b) * 32;
            auto ex = [](int v) { return std::max(0, v - 1); };
            e += kClauseClash * (ex(cj[wa + rc] - 1) - ex(cj[wa + rc]) + ex(cj[wa + rd] + 1) - ex(cj[wa + rd]));
            e += kClauseClash * (ex(cj[wb + rd] - 1) - ex(cj[wb + rd]) + ex(cj[wb + rc] + 1) - ex(cj[wb + rc]));
        }
        return e;
    };
    auto move = [&](int j, int from, int to) {
        for (int i = 0; i < p.length[j]; i++) {
            cnt[(size_t)from * 32 + bank[p.start[j] + i]]--;
            cnt[(size_t)to * 32 + bank[p.start[j] + i]]++;
        }
        cj[(size_t)warp(from) * 32 + (j & 31)]--;
        cj[(size_t)warp(to) * 32 + (j & 31)]++;
    };
    std::vector<std::pair<int, int>> where(p.m);  // clause -> (group, position)
    for (int g = 0; g < G; g++)
        for (int u = 0; u < (int)groups[g].size(); u++) where[groups[g][u]] = {g, u};
    int cursor = 0;
    for (int pass = 0; pass < 2; pass++) {
        bool changed = false;
        for (int a = 0; a < G; a++) {
            for (int guard = 0; guard < 4 * lanes && bad(a); guard++) {
                bool done = false;
                for (int u = 0; u < (int)groups[a].size() && !done; u++) {
                    const int c = groups[a][u];
                    if (!involved(c, a)) continue;
                    for (int t = 0; t < std::min(p.m, 512) && !done; t++) {
                        const int d = (cursor + t) % p.m;
                        const int b = where[d].first;
                        if (b == a || delta(c, a, d, b) >= 0) continue;
                        const int v = where[d].second;
                        move(c, a, b);
                        move(d, b, a);
                        groups[a][u] = d;
                        groups[b][v] = c;
                        where[c] = {b, v};
                        where[d] = {a, u};
                        cursor = (cursor + t + 1) % p.m;
                        done = changed = true;
                    }
                }
                if (!done) break;
            }
        }
        if (!changed) break;
    }
}

// Pair layout: make the public clause indices of every warp distinct mod 32 by swapping
// a repeated clause with a clause of another warp that has the same sorted bank tuple
// (so every group keeps its bank counts) and whose index is free here, while the
// repeated one's index is free there.
void fix_clause_banks(const HostProblem& p, const std::vector<int32_t>& bank, int k,
                      std::vector<std::vector<int32_t>>& groups) {
    const int G = (int)groups.size();
    auto key_of = [&](int j) {
        int b[16];
        const int len = std::min(p.length[j], 16);
        for (int i = 0; i < len; i++) b[i] = bank[p.start[j] + i];
        std::sort(b, b + len);
        uint64_t key = (uint64_t)len;
        for (int i = 0; i < len; i++) key = key * 33 + (uint64_t)b[i];
        return key;
    };
    std::unordered_map<uint64_t, std::vector<int32_t>> by_key;
    std::vector<std::pair<int, int>> where(p.m);
    std::vector<int32_t> cj((size_t)(G / 2 + 1) * 32, 0);
    for (int g = 0; g < G; g++)
        for (int u = 0; u < (int)groups[g].size(); u++) {
            const int j = groups[g][u];
            where[j] = {g, u};
            by_key[key_of(j)].push_back(j);
            cj[(size_t)(g / 2) * 32 + (j & 31)]++;
        }
    (void)k;
    for (int w = 0; 2 * w < G; w++) {
        for (int g = 2 * w; g < std::min(G, 2 * w + 2); g++) {
            for (int u = 0; u < (int)groups[g].size(); u++) {
                const int c = groups[g][u];
                if (cj[(size_t)w * 32 + (c & 31)] <= 1) continue;
                for (int d : by_key[key_of(c)]) {
                    const int h = where[d].first, wb = h / 2;
                    if (wb == w || cj[(size_t)w * 32 + (d & 31)] != 0) continue;
                    if (cj[(size_t)wb * 32 + (c & 31)] - ((d & 31) == (c & 31)) != 0) continue;
                    const int v = where[d].second;
                    cj[(size_t)w * 32 + (c & 31)]--;
                    cj[(size_t)w * 32 + (d & 31)]++;
                    cj[(size_t)wb * 32 + (d & 31)]--;
                    cj[(size_t)wb * 32 + (c & 31)]++;
                    groups[g][u] = d;
                    groups[h][v] = c;
                    where[d] = {g, u};
                    where[c] = {h, v};
                    break;
                }
            }
        }
    }
}

// Bank-aware grouping when literals may be reordered: a group of `lanes` clauses is
// conflict-free in every literal slot as soon as no bank carries more than k of its
// literals (colour_group then finds the slots), so the grouping only balances bank
// counts.  Clauses are taken in a shuffled order by first fit (within a search
// window) until three lanes are left; those are filled by an exact cover of the
// remaining bank capacity from an index of clauses by sorted bank tuple (k <= 4, all
// clauses of length k), else by the least-overfull candidates.  Pair layout: 16-lane
// groups over 16 bank pairs, and the 32 clauses of a warp also take distinct public
// indices mod 32.  Deterministic (fixed seed).
void schedule_balanced(const HostProblem& p, PackedProblem& q, bool pairs,
                       std::vector<std::vector<int8_t>>& order) {
    const int m = p.m, k = p.k;
    const int lanes = pairs ? 16 : 32;
    order.assign(m, {});
    q.cperm.resize(m);
    q.icperm.resize(m);
    std::vector<int32_t> bank(p.storage.size());
    for (size_t i = 0; i < p.storage.size(); i++) bank[i] = q.iperm[std::abs(p.storage[i]) - 1] & (lanes - 1);
    std::vector<int32_t> rem(m);
    for (int j = 0; j < m; j++) rem[j] = j;
    uint64_t rng = 0x9E3779B97F4A7C15ull;
    for (int j = m - 1; j > 0; j--) {
        rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17;
        std::swap(rem[j], rem[rng % (uint64_t)(j + 1)]);
    }
    // index of full-length clauses by their sorted bank tuple (5 bits per bank)
    const bool exact = k <= 4;
    auto key_of = [&](const int* b) {
        uint32_t key = 0;
        for (int i = 0; i < k; i++) key |= (uint32_t)b[i] << (5 * i);
        return key;
    };
    std::unordered_map<uint32_t, std::vector<int32_t>> by_key;
    if (exact)
        for (int t = m - 1; t >= 0; t--) {  // reversed: lists are consumed from the back
            const int j = rem[t];
            if (p.length[j] != k) continue;
            int b[4];
            for (int i = 0; i < k; i++) b[i] = bank[p.start[j] + i];
            std::sort(b, b + k);
            by_key[key_of(b)].push_back(j);
        }
    std::vector<char> taken(m, 0);
    const size_t kScanWindow = 4096;
    const int kFillWindow = 1024;
    const int kEnd = 3;  // lanes left to the exact cover
    // a repeated clause bank costs four extra wavefronts (two loads, two stores of a_m)
    // against two for a literal bank (one gather, one store): weigh it accordingly
    const int kClauseClash = 3;
    int cnt[32];
    uint32_t used_clause = 0;
    auto over = [&](int j) {  // literals beyond k per bank if j joins, + clause-bank clash
        int add[32] = {0}, o = pairs ? kClauseClash * (int)((used_clause >> (j & 31)) & 1u) : 0;
        for (int i = 0; i < p.length[j]; i++) {
            const int b = bank[p.start[j] + i];
            if (cnt[b] + ++add[b] > k) o++;
        }
        return o;
    };
    std::vector<int32_t> keep, members;
    auto take = [&](int j) {
        for (int i = 0; i < p.length[j]; i++) cnt[bank[p.start[j] + i]]++;
        used_clause |= 1u << (j & 31);
        members.push_back(j);
        taken[j] = 1;
    };
    auto untake = [&](int j) {
        for (int i = 0; i < p.length[j]; i++) cnt[bank[p.start[j] + i]]--;
        used_clause &= ~(1u << (j & 31));
        members.pop_back();
        taken[j] = 0;
    };
    // a free clause with bank tuple `b` (sorted) that respects the clause banks
    auto find = [&](const int* b) -> int {
        auto it = by_key.find(key_of(b));
        if (it == by_key.end()) return -1;
        auto& v = it->second;
        while (!v.empty() && taken[v.back()]) v.pop_back();
        for (int t = (int)v.size() - 1; t >= 0 && t >= (int)v.size() - 64; t--)
            if (!taken[v[t]] && !(pairs && ((used_clause >> (v[t] & 31)) & 1u))) return v[t];
        return -1;
    };
    // exact cover of the capacity left (k - cnt[b] per bank) by r full-length clauses
    std::function<bool(int)> cover = [&](int r) -> bool {
        if (r == 0) return true;
        int b0 = -1;
        for (int b = 0; b < lanes && b0 < 0; b++)
            if (cnt[b] < k) b0 = b;
        if (b0 < 0) return false;
        int tup[4];
        tup[0] = b0;
        // choose tup[1..k-1] non-decreasing from the capacity left after b0
        std::function<bool(int, int)> pick = [&](int pos, int from) -> bool {
            if (pos == k) {
                const int j = find(tup);
                if (j < 0) return false;
                take(j);
                if (cover(r - 1)) return true;
                untake(j);
                return false;
            }
            for (int b = from; b < lanes; b++) {
                int used = 0;
                for (int i = 0; i < pos; i++) used += tup[i] == b;
                if (cnt[b] + used >= k) continue;
                tup[pos] = b;
                if (pick(pos + 1, b)) return true;
            }
            return false;
        };
        return pick(1, b0);
    };
    std::vector<std::vector<int32_t>> groups, gb;
    std::vector<std::vector<int8_t>> slots;
    int out = 0;
    while (!rem.empty()) {
        used_clause = 0;
        for (int h = 0; h < 32 / lanes && !rem.empty(); h++) {
            std::fill(cnt, cnt + 32, 0);
            members.clear();
            keep.clear();
            size_t scanned = 0;
            const int stop = exact ? lanes - kEnd : lanes;
            for (int j : rem) {
                if (taken[j]) continue;
                if ((int)members.size() < stop && scanned++ < kScanWindow && over(j) == 0) take(j);
                else keep.push_back(j);
            }
            const int left = lanes - (int)members.size();
            bool full = true;
            for (int u : members) full = full && p.length[u] == k;
            if (exact && full && left <= kEnd && left <= (int)keep.size()) cover(left);
            for (size_t t = 0; t < keep.size(); t++)
                if (taken[keep[t]]) { keep[t] = keep.back(); keep.pop_back(); t--; }
            while ((int)members.size() < lanes && !keep.empty()) {
                int best = 0, bo = 1 << 30;
                for (int c = 0; c < (int)keep.size() && c < kFillWindow && bo > 0; c++) {
                    const int o = over(keep[c]);
                    if (o < bo) { bo = o; best = c; }
                }
                const int j = keep[best];
                keep.erase(keep.begin() + best);
                take(j);
            }
            rem.swap(keep);
            groups.push_back(members);
            out += (int)members.size();
        }
    }
    repair_groups(p, bank, lanes, k, pairs, groups);
    if (pairs) fix_clause_banks(p, bank, k, groups);
    out = 0;
    for (const auto& g : groups) {
        gb.assign(g.size(), {});
        for (size_t u = 0; u < g.size(); u++)
            for (int l = 0; l < p.length[g[u]]; l++) gb[u].push_back(bank[p.start[g[u]] + l]);
        colour_group(gb, lanes, k, slots);
        for (size_t u = 0; u < g.size(); u++) {
            order[out] = slots[u];
            q.cperm[out] = g[u];
            out++;
        }
    }
    for (int mi = 0; mi < m; mi++) q.icperm[q.cperm[mi]] = mi;
    long waves = 0;
    for (int g = 0; g < m; g += lanes)
        for (int qq = 0; qq < std::min(k, 16); qq++) {
            int c[32] = {0}, mx = 0;
            for (int mi = g; mi < std::min(m, g + lanes); mi++) {
                const int li = order[mi][qq];
                if (li >= 0) mx = std::max(mx, ++c[bank[p.start[q.cperm[mi]] + li]]);
            }
            waves += std::max(mx, 1);
        }
    q.bank_wavefronts = waves;
}

}  // namespace

bool pack_parts(const HostProblem& p, const PackedProblem& q, int nparts, PartLayout& out) {
    out = PartLayout();
    if (p.n >= 8191 || p.k > 16 || nparts < 1 || (int)q.iperm.size() != p.n) return false;
    const int n = p.n, m = p.m, k = p.k, ns = (n + 31) / 32;
    if (nparts == 1) {
        // one part is the FP32 packing itself: its clause grouping, literal order and slots
        if (q.nslots >= (1 << 17)) return false;
        out.nparts = 1;
        out.max_slots = q.nslots;
        out.c0 = {0, m};
        out.srow = q.srow;
        out.cperm = q.cperm;
        out.icperm = q.icperm;
        out.cnt.assign(n, 0);
        out.words.assign((size_t)m * k, 0);
        for (int mi = 0; mi < m; mi++)
            for (int qq = 0; qq < k; qq++) {
                const size_t idx = (size_t)qq * q.mp + mi;
                const uint32_t v = q.litw[idx] & 0x7fffffffu;
                if ((int)v < n) out.cnt[v]++;
                out.words[(size_t)mi * k + qq] = (q.litw[idx] & 0x80000000u) | (q.slotw[idx] << 13) | v;
            }
        return true;
    }
    out.nparts = nparts;
    out.c0.assign(nparts + 1, 0);
    out.srow.assign((size_t)nparts * (ns + 1), 0);
    out.cnt.assign((size_t)nparts * n, 0);
    out.cperm.resize(m);
    out.icperm.resize(m);
    out.words.assign((size_t)m * k, 0);
    std::vector<int32_t> slot_of(p.storage.size(), 0);
    int mi0 = 0;
    for (int pp = 0; pp < nparts; pp++) {
        const int j0 = (int)((long long)m * pp / nparts), j1 = (int)((long long)m * (pp + 1) / nparts);
        out.c0[pp] = mi0;
        // occurrences per internal variable in this part, SELL rows per slice
        uint16_t* cnt = out.cnt.data() + (size_t)pp * n;
        for (int j = j0; j < j1; j++)
            for (int i = 0; i < p.length[j]; i++) {
                const int v = q.iperm[std::abs(p.storage[p.start[j] + i]) - 1];
                if (cnt[v] == 0xFFFF) return false;
                cnt[v]++;
            }
        int32_t* srow = out.srow.data() + (size_t)pp * (ns + 1);
        for (int g = 0; g < ns; g++) {
            int w = 0;
            for (int l = 0; l < 32 && g * 32 + l < n; l++) w = std::max(w, (int)cnt[g * 32 + l]);
            srow[g + 1] = srow[g] + w;
        }
        const int nslots = srow[ns] * 32;
        if (nslots >= (1 << 17)) { out = PartLayout(); return false; }
        out.max_slots = std::max(out.max_slots, nslots);
        std::vector<int32_t> rank(n, 0);
        for (int j = j0; j < j1; j++)
            for (int i = 0; i < p.length[j]; i++) {
                const int v = q.iperm[std::abs(p.storage[p.start[j] + i]) - 1];
                slot_of[p.start[j] + i] = (srow[v >> 5] + rank[v]++) * 32 + (v & 31);
            }
        // bank-aware warp grouping of this part's clauses (banks: internal variable mod 32)
        HostProblem sub;
        sub.n = n;
        sub.k = k;
        for (int j = j0; j < j1; j++) {
            sub.start.push_back((int32_t)sub.storage.size());
            sub.length.push_back(p.length[j]);
            for (int i = 0; i < p.length[j]; i++) sub.storage.push_back(p.storage[p.start[j] + i]);
        }
        sub.m = j1 - j0;
        PackedProblem tq;
        tq.iperm = q.iperm;
        std::vector<std::vector<int8_t>> order;
        if (sub.m > 0) schedule_balanced(sub, tq, false, order);
        for (int t = 0; t < sub.m; t++) {
            const int j = j0 + tq.cperm[t], mi = mi0 + t;
            out.cperm[mi] = j;
            out.icperm[j] = mi;
            for (int qq = 0; qq < k; qq++) {
                const int li = qq < (int)order[t].size() ? order[t][qq] : -1;
                uint32_t w;
                if (li < 0) {
                    w = ((uint32_t)nslots << 13) | (uint32_t)n;  // sentinel: spin -1, trash slot
                } else {
                    const int lit = p.storage[p.start[j] + li];
                    const uint32_t v = (uint32_t)q.iperm[std::abs(lit) - 1];
                    w = (lit < 0 ? 0x80000000u : 0u) | ((uint32_t)slot_of[p.start[j] + li] << 13) | v;
                }
                out.words[(size_t)mi * k + qq] = w;
            }
        }
        mi0 += sub.m;
    }
    out.c0[nparts] = mi0;
    return true;
}

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
    // Inside a slice the lane order is free (slice widths depend only on membership):
    // give the slice's variables, heaviest first, to the lanes whose banks (lane mod
    // 32) carry the fewest literals so far, so every bank ends up with about M k / 32
    // literals -- what the bank-aware clause grouping needs to be conflict-free.
    {
        std::vector<long> load(32, 0);
        std::vector<int32_t> lane(32), vars(32);
        const int ns = (p.n + 31) / 32;
        for (int t = 0; t < ns; t++) {  // the partial last slice first: its lanes are fixed
            const int g = (t + ns - 1) % ns;
            const int w = std::min(32, p.n - g * 32);
            for (int l = 0; l < w; l++) { lane[l] = l; vars[l] = q.perm[g * 32 + l]; }
            std::stable_sort(lane.begin(), lane.begin() + w, [&](int a, int b) { return load[a] < load[b]; });
            for (int i = 0; i < w; i++) {
                q.perm[g * 32 + lane[i]] = vars[i];
                load[lane[i]] += degree[vars[i]];
            }
        }
    }
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
        if (permute_literals && p.k <= 16)
            schedule_balanced(p, q, mode == kPackF32Pair, order);
        else
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
        for (int qq = 0; qq < (int)order[mi].size(); qq++) {  // slot qq; -1 = sentinel
            if (order[mi][qq] < 0) continue;
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
