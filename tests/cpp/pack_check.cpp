// Structural checks of the device packing (analogsat_b200/csrc/as_problem.cpp) on random
// instances, all three packing modes: every internal clause carries exactly its public
// literals (sign and variable), every literal owns one distinct contribution slot in
// its variable's SELL row, rows follow the public (clause, literal) order, the
// permutations are inverse pairs, and the bank-group diagnostics are at least ideal;
// and the clause-parts layout of the lean kernel's global-rows form.
// Built with g++ against the host sources only (no CUDA).  Exit code 0 = all good.
#include "../../analogsat_b200/csrc/as_problem.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace asb;

static uint64_t rng_state = 0x1234567887654321ull;
static uint32_t rnd(uint32_t n) {
    rng_state ^= rng_state << 13;
    rng_state ^= rng_state >> 7;
    rng_state ^= rng_state << 17;
    return (uint32_t)(rng_state % n);
}

static int check(const HostProblem& hp, int mode) {
    const PackedProblem q = pack(hp, mode);
    const int n = q.n, m = q.m, k = q.k;
    for (int v = 0; v < n; v++)
        if (q.iperm[q.perm[v]] != v) return 10;
    for (int c = 0; c < m; c++)
        if (q.icperm[q.cperm[c]] != c) return 11;
    std::vector<int> slot_owner(q.nslots + 1, -1);
    std::vector<std::vector<std::pair<int, int>>> rows(n);  // var -> (row, public clause)
    for (int mi = 0; mi < m; mi++) {
        const int j = q.cperm[mi];
        std::vector<long> want, got;
        for (int i = 0; i < hp.length[j]; i++) {
            const int lit = hp.storage[hp.start[j] + i];
            want.push_back(2L * q.iperm[std::abs(lit) - 1] + (lit < 0));
        }
        for (int s = 0; s < k; s++) {
            const uint32_t w = q.litw[(size_t)s * q.mp + mi];
            const uint32_t v = w & 0x7fffffffu, slot = q.slotw[(size_t)s * q.mp + mi];
            if ((int)v == n) {  // sentinel: trash slot, positive
                if (slot != (uint32_t)q.nslots || (w >> 31)) return 12;
                continue;
            }
            if ((int)v > n || slot >= (uint32_t)q.nslots || slot_owner[slot] >= 0) return 13;
            slot_owner[slot] = mi;
            if ((int)(slot & 31) != (int)(v & 31)) return 14;
            const int g = (int)v >> 5, row = (int)(slot >> 5);
            if (row < q.srow[g] || row >= q.srow[g + 1]) return 15;
            rows[v].push_back({row, j});
            got.push_back(2L * v + (w >> 31));
            if (q.compact) {
                const uint32_t cw = q.lit[(size_t)s * q.mp + mi];
                if (cw != ((w & 0x80000000u) | (v << 16) | slot)) return 16;
            }
        }
        std::sort(want.begin(), want.end());
        std::sort(got.begin(), got.end());
        if (want != got) return 17;
    }
    for (int v = 0; v < n; v++) {  // rows in public clause order, from the slice's first row
        auto r = rows[v];
        std::sort(r.begin(), r.end());
        for (size_t t = 0; t < r.size(); t++) {
            if (r[t].first != q.srow[v >> 5] + (int)t) return 18;
            if (t && r[t].second < r[t - 1].second) return 19;
        }
    }
    if (q.compact && m >= 32) {
        const int lanes = mode == kPackF32Pair ? 16 : 32;
        if (q.bank_wavefronts < (long)std::min(k, 16) * ((m + lanes - 1) / lanes)) return 20;
    }
    return 0;
}

// Clause parts (pack_parts): every public clause once, parts as public-index ranges,
// each literal one distinct slot of its part's buffer in its variable's SELL column,
// rows in public clause order within the part, occurrence counts consistent.
static int check_parts(const HostProblem& hp, int nparts) {
    const PackedProblem q = pack(hp, kPackF32);
    PartLayout L;
    if (!pack_parts(hp, q, nparts, L)) return hp.n >= 8191 ? 0 : 30;
    const int n = q.n, m = q.m, k = q.k, ns = (n + 31) / 32;
    if (L.nparts != nparts || (int)L.c0.size() != nparts + 1 || L.c0[nparts] != m) return 31;
    for (int c = 0; c < m; c++)
        if (L.icperm[L.cperm[c]] != c) return 32;
    for (int pp = 0; pp < nparts; pp++) {
        const int j0 = (int)((long long)m * pp / nparts), j1 = (int)((long long)m * (pp + 1) / nparts);
        const int32_t* srow = L.srow.data() + (size_t)pp * (ns + 1);
        const int nslots = srow[ns] * 32;
        if (nslots > L.max_slots) return 33;
        std::vector<int> owner(nslots + 1, -1);
        std::vector<std::vector<std::pair<int, int>>> rows(n);
        std::vector<int> cnt(n, 0);
        for (int mi = L.c0[pp]; mi < L.c0[pp + 1]; mi++) {
            const int j = L.cperm[mi];
            if (j < j0 || j >= j1) return 34;
            std::vector<long> want, got;
            for (int i = 0; i < hp.length[j]; i++) {
                const int lit = hp.storage[hp.start[j] + i];
                want.push_back(2L * q.iperm[std::abs(lit) - 1] + (lit < 0));
            }
            for (int s = 0; s < k; s++) {
                const uint32_t w = L.words[(size_t)mi * k + s];
                const int v = (int)(w & 0x1FFFu), slot = (int)((w >> 13) & 0x1FFFFu);
                if (v == n) {
                    if (slot != nslots || (w >> 31)) return 35;
                    continue;
                }
                if (v > n || slot >= nslots || owner[slot] >= 0 || (slot & 31) != (v & 31)) return 36;
                owner[slot] = mi;
                const int row = slot >> 5;
                if (row < srow[v >> 5] || row >= srow[(v >> 5) + 1]) return 37;
                rows[v].push_back({row, j});
                cnt[v]++;
                got.push_back(2L * v + (w >> 31));
            }
            std::sort(want.begin(), want.end());
            std::sort(got.begin(), got.end());
            if (want != got) return 38;
        }
        for (int v = 0; v < n; v++) {
            if (cnt[v] != (int)L.cnt[(size_t)pp * n + v]) return 39;
            auto r = rows[v];
            std::sort(r.begin(), r.end());
            for (size_t t = 0; t < r.size(); t++) {
                if (r[t].first != srow[v >> 5] + (int)t) return 40;
                if (t && r[t].second < r[t - 1].second) return 41;
            }
        }
    }
    return 0;
}

int main() {
    int cases = 0;
    for (int trial = 0; trial < 40; trial++) {
        const int k = 2 + (int)rnd(4);                  // 2..5
        const int n = 8 + (int)rnd(trial < 30 ? 400 : 3000);
        const int m = 1 + (int)rnd(5 * n);
        const bool mixed = trial % 3 == 0;
        std::vector<int32_t> lits, lens;
        for (int c = 0; c < m; c++) {
            const int len = mixed ? 1 + (int)rnd(k) : k;
            const int vlen = std::min(len, n);
            std::vector<int> vs;
            while ((int)vs.size() < vlen) {
                const int v = 1 + (int)rnd(n);
                if (std::find(vs.begin(), vs.end(), v) == vs.end()) vs.push_back(v);
            }
            for (int v : vs) lits.push_back(rnd(2) ? v : -v);
            lens.push_back(vlen);
        }
        HostProblem hp;
        hp.add_clauses(lits.data(), lens.data(), (int)lens.size());
        for (int mode : {kPackReference, kPackF32, kPackF32Pair}) {
            const int r = check(hp, mode);
            cases++;
            if (r) {
                std::printf("FAIL trial %d mode %d n %d m %d k %d: code %d\n", trial, mode, n, m, k, r);
                return r;
            }
        }
        for (int np : {1, 2, 3}) {
            const int r = check_parts(hp, np);
            cases++;
            if (r) {
                std::printf("FAIL trial %d parts %d n %d m %d k %d: code %d\n", trial, np, n, m, k, r);
                return r;
            }
        }
    }
    std::printf("pack ok %d\n", cases);
    return 0;
}
