// Lean FP32 persistent solver (shared-memory mode, plain CTDS right-hand side).
//
// The same integrator, counters and early-exit rules as solve_kernel (SatSolver::DoSolve
// + CpuRungeKutta::Step/rkqs/rkck + CpuSat::GetDerivatives/GetClauseViolationCount:
// AnalogSAT/solver/SatSolver.h:273-355, AnalogSAT/cpu_sat/CpuRungeKutta.cpp:66-100,
// 181-267, AnalogSAT/cpu_sat/CpuSat.cpp:65-94,136-173,199-241) and the same FP32
// arithmetic as its log-space FP32 path (bit-identical results), with the instruction
// count per clause cut down -- the shared-memory solver is issue bound, so its RHS rate
// is the inverse of the instructions it executes per clause and stage:
//
//  * Literal words carry shared-memory addressing (DevInstance::flit): bits 0-13 the
//    byte offset of the literal's spin from the spin base (aligned to a power of two
//    at least the spins' size, so base | offset is the address), bits 14-30 the index
//    of its contribution slot, bit 31 the sign.  The spins are held twice, the second
//    copy negated (neg_spin_base), and a negated literal's word points into it: a spin
//    gather is one logic operation and one load, with no sign flip.
//  * The clause arithmetic folds its power-of-two scalings (fast_clause), as the
//    general kernel's FP32 log-space path does.
//  * Each stage's variable phase also forms the next stage's spin input, and an
//    accepted step's copy of the clause rows happens in the next stage 1's clause
//    loop; the error max is an integer redux (lean_max_then) and an accepted step's
//    next step size is formed in the next stage 1 (settle_h).
//  * Literal words are blocked by 32 clauses ([m / 32][q][m % 32]), so a clause's K
//    words are loads at immediate offsets from one pointer that advances once per
//    clause, and a warp's 32 clauses load each word as one 128-byte line.
//  * The six RK vectors of an element are interleaved, [e][X, K1, K2, K3, K4, K5]
//    (24 bytes per element): a stage input is one row address and 64-bit loads at
//    immediate offsets (a 16-lane half-warp at a 24-byte stride covers all 32 banks
//    once, so the pairs load without bank conflicts).  The stage-6 candidate state is
//    written into K2's place and copied into X's on acceptance (each element by its
//    own thread, no barrier).
//  * No model branches: instances with the tanh variant or a bias term use
//    solve_kernel.
//  * ROWS_G: the RK rows live in a per-CTA slab of global memory (L2-resident while
//    the slabs in flight fit), blocked by 32 elements so that every row access of a
//    warp is one coalesced line per field, and only the spins and the contribution
//    slots in shared memory -- the gathers and scatters stay on chip.  With the
//    clauses in parts (each part's contributions summed before the next part reuses
//    the slots) this takes instances up to N < 8191, where the all-shared layout
//    stops at N of about 1,240.
// The bank-aware clause grouping of the FP32 packing applies unchanged: a literal's
// spin and its slot both sit in bank (internal variable mod 32).
#pragma once

#include <type_traits>

#include "as_kernels.cuh"

namespace asb {

// Shared-memory byte offsets of the lean layout for an instance, and whether its
// literal words can carry them (spin offsets below 16 KB, slot indices below 2^17).
// bytes: shared memory of the all-shared form (rows on chip); cs_off_g: where the
// global-rows form's slots start (one spin copy).
// The all-shared form holds the spins twice, s_0..s_N (s_N the sentinel) and, from the
// next multiple of 32 floats (neg_spin_base, so -s_v sits in s_v's bank), -s_0..-s_N: a
// negated literal's word points at its negated spin and a gather needs no sign flip.
// Both copies sit at a shared address aligned to spin_align (the smallest power of two
// >= their bytes), so a spin's address is that base OR the byte offset of its literal
// word: one logic operation.  bytes counts the worst-case padding.  The global-rows
// form holds one copy; its slots start at cs_off_g.
__host__ __device__ inline int neg_spin_base(int n) { return (n + 1 + 31) & ~31; }
__host__ __device__ inline uint32_t spin_align(int n) {
    uint32_t a = 128;
    while (a < 4u * (uint32_t)(neg_spin_base(n) + n + 1)) a <<= 1;
    return a;
}
struct FastLayout {
    bool ok = false;
    int cs_off = 0, rows_off = 0, cs_off_g = 0;
    size_t bytes = 0;
};
__host__ __device__ inline FastLayout fast_layout(int n, int m, int nslots) {
    FastLayout L;
    L.cs_off = ((4 * (neg_spin_base(n) + n + 1)) + 127) / 128 * 128;  // a multiple of 128 B keeps slot banks
    L.cs_off_g = ((4 * (n + 1)) + 127) / 128 * 128;
    const long long cs_end = (long long)L.cs_off + 4ll * (nslots + 1);
    L.rows_off = (int)((cs_end + 15) / 16 * 16);
    L.bytes = (size_t)L.rows_off + 24ull * (size_t)(n + m) + spin_align(n) - 16;
    L.ok = 4ll * (neg_spin_base(n) + n + 1) <= 16384 && nslots < (1 << 17);
    return L;
}

// The lean kernels' literal words are blocked by 32 clauses, [c / 32][q][c % 32]: the
// 32 consecutive clauses of a warp load word q as one 128-byte line (clause-major words
// would spread it over 12 or 16 sectors).  lean_words: the words of m clauses, padded.
__host__ __device__ inline size_t lean_word_index(int c, int q, int k) {
    return (size_t)(c >> 5) * 32 * k + 32 * q + (c & 31);
}
__host__ __device__ inline size_t lean_words(int m, int k) { return (size_t)((m + 31) & ~31) * k; }

__device__ __forceinline__ uint32_t ld_lit(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::evict_last.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// Shared-memory accesses by 32-bit shared-window address (the dynamic shared memory's
// base plus a byte offset), so no address arithmetic is wider than 32 bits.
__device__ __forceinline__ float lds(uint32_t a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ float2 lds2(uint32_t a) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ void sts(uint32_t a, float v) {
    asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}

// The entries of one element's interleaved row that stage S reads (X, K1..K_{S-1}),
// in 64-bit loads.
struct Row6 {
    float x = 0.f, k1 = 0.f, k2 = 0.f, k3 = 0.f, k4 = 0.f, k5 = 0.f;
};
// Where the interleaved rows live: shared memory (32-bit shared-window addresses) or a
// per-CTA global slab.  at(e) is element e's row; ld/ld2/st take the float index in it.
template <bool G> struct RowStore;
template <> struct RowStore<false> {
    using Ref = uint32_t;
    uint32_t base;
    __device__ __forceinline__ Ref at(int e) const { return base + 24u * (uint32_t)e; }
    __device__ __forceinline__ static Ref advance(Ref r, int elems) { return r + 24u * (uint32_t)elems; }
    __device__ __forceinline__ static float ld(Ref r, int i) { return lds(r + 4u * i); }
    __device__ __forceinline__ static float2 ld2(Ref r, int i) { return lds2(r + 4u * i); }
    __device__ __forceinline__ static void st(Ref r, int i, float v) { sts(r + 4u * i, v); }
};
// In global memory the rows are blocked by 32 elements, [e / 32][X, K1..K5][e % 32]: a
// warp's 32 consecutive elements read or write one field as one 128-byte line (an
// interleaved 24-byte row would spread a warp's 32-bit store over 24 sectors).
// advance() takes a multiple of 32 elements.
template <> struct RowStore<true> {
    using Ref = float*;
    float* base;
    __device__ __forceinline__ Ref at(int e) const { return base + 192ll * (e >> 5) + (e & 31); }
    __device__ __forceinline__ static Ref advance(Ref r, int elems) { return r + 6ll * elems; }
    __device__ __forceinline__ static float ld(Ref r, int i) { return r[32 * i]; }
    __device__ __forceinline__ static float2 ld2(Ref r, int i) { return make_float2(r[32 * i], r[32 * i + 32]); }
    __device__ __forceinline__ static void st(Ref r, int i, float v) { r[32 * i] = v; }
};
// First row of the clauses: right after the variables' rows in shared memory; in a
// global slab at the next 32-element block, so a warp's clause rows share blocks.
template <bool G>
__host__ __device__ inline int row_clause_base(int n) { return G ? (n + 31) & ~31 : n; }

template <int S, typename R>
__device__ __forceinline__ Row6 load_row(typename R::Ref r) {
    Row6 o;
    if constexpr (S == 1) {
        o.x = R::ld(r, 0);
    } else {
        const float2 a = R::ld2(r, 0);
        o.x = a.x; o.k1 = a.y;
        if constexpr (S == 3) o.k2 = R::ld(r, 2);
        if constexpr (S >= 4) {
            const float2 b = R::ld2(r, 2);
            o.k2 = b.x; o.k3 = b.y;
        }
        if constexpr (S == 5) o.k4 = R::ld(r, 4);
        if constexpr (S == 6) {
            const float2 c = R::ld2(r, 4);
            o.k4 = c.x; o.k5 = c.y;
        }
    }
    return o;
}
// A clause row at stage 1: after an accepted step its new state still sits in slot 2
// (the accepted step's copy of the clause rows is done here, by the owning thread,
// where the row is read anyway).
template <int S, typename R>
__device__ __forceinline__ Row6 load_clause_row(typename R::Ref r, bool from_candidate) {
    if constexpr (S == 1) {
        if (from_candidate) {
            Row6 o;
            o.x = R::ld(r, 2);
            R::st(r, 0, o.x);
            return o;
        }
    }
    return load_row<S, R>(r);
}
template <int S>
__device__ __forceinline__ float row_input(const Row6& o, float h) {
    return stage_in<S, float>(o.x, o.k1, o.k2, o.k3, o.k4, o.k5, h);
}
// Puts the stage-S derivative into its place of a row read for stage S, which then
// holds what stage S + 1 reads.
template <int S>
__device__ __forceinline__ void set_k(Row6& o, float k) {
    if constexpr (S == 1) o.k1 = k;
    if constexpr (S == 2) o.k2 = k;
    if constexpr (S == 3) o.k3 = k;
    if constexpr (S == 4) o.k4 = k;
    if constexpr (S == 5) o.k5 = k;
}

// 1 - c s for a literal word (the sign bit flips s: 1 - (-s) = 1 + s), as clause_phase.
__device__ __forceinline__ float lit_factor(uint32_t sb, uint32_t mask, uint32_t w) {
    return 1.0f - lds(sb | (w & mask));  // the word points at -s for a negated literal
}

// Clause phase of one clause (K literals, FP32, log-space weights): spin gathers,
// K_m, the leave-one-out products in CpuProdWrapper order, contributions into their
// slots; returns du_m = K_m^2 / ln 2.  Same operations as clause_phase<float, true, K>,
// with its power-of-two scalings folded: with P = f_0 f_1 .. f_{K-1}, K_m = knorm P and
// 2 r = 2 (K_m knorm) a_m = P (a_m 2 knorm^2), du_m = (P P)(knorm^2 / ln 2) -- the same
// roundings (a power-of-two factor scales a rounded product exactly).  am2 = a_m 2
// knorm^2, duc = knorm^2 / ln 2.
template <int K>
__device__ __forceinline__ float fast_clause(uint32_t sb, uint32_t mask, uint32_t cs0, const uint32_t* lp, float am2,
                                             float duc) {
    uint32_t w[K];
    float f[K];
#pragma unroll
    for (int q = 0; q < K; q++) w[q] = ld_lit(lp + 32 * q);
    float P = 0.0f;
#pragma unroll
    for (int q = 0; q < K; q++) {
        f[q] = lit_factor(sb, mask, w[q]);
        P = q == 0 ? f[0] : P * f[q];
    }
    const float r2 = P * am2;
#pragma unroll
    for (int q = 0; q < K; q++) {
        float prod = 1.0f;
        bool first = true;
#pragma unroll
        for (int l = 0; l < K; l++) {
            if (l != q) {
                prod = first ? f[l] : prod * f[l];
                first = false;
            }
        }
        const float rr = r2 * prod;  // (2r) prod == 2 (r prod) above the subnormals
        sts(cs0 + 4u * ((w[q] >> 14) & 0x1FFFFu), __int_as_float(__float_as_int(rr) ^ (int)(w[q] & 0x80000000u)));
    }
    return (P * P) * duc;
}

// The same on a clause-parts word (bits 0-12 internal variable, 13-29 slot, 31 sign).
template <int K>
__device__ __forceinline__ float part_clause(uint32_t sm0, uint32_t cs0, const uint32_t* lp, float am2,
                                             float duc) {
    uint32_t w[K];
    float f[K];
#pragma unroll
    for (int q = 0; q < K; q++) w[q] = ld_lit(lp + 32 * q);
    float P = 0.0f;
#pragma unroll
    for (int q = 0; q < K; q++) {
        const float sv = lds(sm0 + 4u * (w[q] & 0x1FFFu));
        f[q] = 1.0f - __int_as_float(__float_as_int(sv) ^ (int)(w[q] & 0x80000000u));
        P = q == 0 ? f[0] : P * f[q];
    }
    const float r2 = P * am2;
#pragma unroll
    for (int q = 0; q < K; q++) {
        float prod = 1.0f;
        bool first = true;
#pragma unroll
        for (int l = 0; l < K; l++) {
            if (l != q) {
                prod = first ? f[l] : prod * f[l];
                first = false;
            }
        }
        const float rr = r2 * prod;
        sts(cs0 + 4u * ((w[q] >> 13) & 0x1FFFFu), __int_as_float(__float_as_int(rr) ^ (int)(w[q] & 0x80000000u)));
    }
    return (P * P) * duc;
}

// Block max of the error ratios, post-processed by thread 0.  The ratios are FP32 and
// never negative (fmaxf from 0 skips NaN), so their bit patterns order like their values
// and a warp's max is one integer redux; the max of floats then converted is the FP64
// max of the converted values, as the general kernel forms it.  red_u is written only
// here, and a block barrier always separates two calls.
template <typename F>
__device__ __forceinline__ double lean_max_then(float em, uint32_t* red_u, double* red_d, F&& fn) {
    const uint32_t v = __reduce_max_sync(0xffffffffu, __float_as_uint(em));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red_u[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const uint32_t x = __reduce_max_sync(0xffffffffu, lane < (int)(blockDim.x >> 5) ? red_u[lane] : 0u);
        if (lane == 0) red_d[33] = fn((double)__uint_as_float(x));
    }
    __syncthreads();
    return red_d[33];
}

__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// ROWS_G = false: rows, spins and slots in shared memory, words flit.  ROWS_G = true:
// rows in the CTA's global slab, spins and slots in shared memory, clauses in parts
// (words plit), each part's contributions summed before the next part reuses the slots.
template <int K, bool ROWS_G>
__global__ void __launch_bounds__(1024, 1) solve_kernel_fast(SolveParams P) {
    using R = RowStore<ROWS_G>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_d[36];
    __shared__ int red_i[33];
    __shared__ uint32_t red_u[32];
    __shared__ int s_unit, s_flag;
    const Grp<1> g;
    const int tid = threadIdx.x, nt = blockDim.x;
    const uint32_t sm0 = (uint32_t)__cvta_generic_to_shared(smem_raw);

    while (true) {
        const int u = g.bcast(&s_unit, tid == 0 ? atomicAdd(P.queue_head, 1) : 0);
        if (u >= P.num_units) break;
        const int pidx = P.unit_inst[u];
        if (g.bcast(&s_flag, tid == 0 && P.stop_on_first ? (atomicAdd(P.inst_solved + pidx, 0) != 0 ? 1 : 0) : 0)) {
            if (tid == 0) {
                UnitResult r;
                r.time = 0.0; r.hdid = 0.0; r.status = SAT_ODE_INTERRUPTED; r.steps = 0; r.attempts = 0;
                r.rhs = 0; r.viol = -1; r.min_viol = -1;
                r.pad0 = r.pad1 = 0;
                P.results[u] = r;
            }
            g.sync();
            continue;
        }
        const DevInstance I = P.inst[pidx];
        const int n = I.n, m = I.m, cb = row_clause_base<ROWS_G>(n);
        // spin base: aligned in the all-shared form (spin_align), the start otherwise
        const uint32_t mask = ROWS_G ? 0u : spin_align(n) - 1u;
        const uint32_t sb = ROWS_G ? sm0 : (sm0 + mask) & ~mask;
        float* const sy = reinterpret_cast<float*>(smem_raw + (sb - sm0));
        const int cso = ROWS_G ? I.cs_off_g : I.cs_off;
        float* const cs = reinterpret_cast<float*>(smem_raw + (sb - sm0) + cso);
        R rs;
        if constexpr (ROWS_G) rs.base = reinterpret_cast<float*>(P.slab) + (long long)blockIdx.x * P.slab_stride;
        else rs.base = sb + (uint32_t)I.rows_off;
        const uint32_t cs0 = sb + (uint32_t)cso;
        // the all-shared form's second, negated spin copy: spin v also at sneg + 4 v
        const uint32_t sneg = sb + 4u * (uint32_t)neg_spin_base(n);
        auto put_spin = [&](int v, float val) {
            sts(sb + 4u * (uint32_t)v, val);
            if constexpr (!ROWS_G) sts(sneg + 4u * (uint32_t)v, -val);
        };
        float* G = reinterpret_cast<float*>(P.states) + P.unit_state[u];
        const float knorm = (float)ldexp(1.0, -I.k);
        const float a2n = 2.0f * knorm * knorm;      // 2 knorm^2 (exact)
        const float duc = knorm * knorm * kInvLn2;   // knorm^2 / ln 2 (exact scaling)
        // the wall-clock deadline (stamped before the launch)
        const unsigned long long deadline = P.deadline ? *P.deadline : 0ull;

        // initial state: public spins to internal order, a -> log2 a
        const int32_t* const icp = ROWS_G ? I.picperm : I.icperm;  // public -> internal clause
        for (int i = tid; i < n; i += nt) R::st(rs.at(__ldg(I.iperm + i)), 0, G[i]);
        for (int j = tid; j < m; j += nt) R::st(rs.at(cb + __ldg(icp + j)), 0, log2f(G[n + j]));
        if constexpr (!ROWS_G)  // padding slots are read as zeros (the parts form reads counts)
            for (int j = tid; j <= I.nslots; j += nt) cs[j] = 0.0f;
        if (tid == 0) put_spin(n, -1.0f);  // sentinel spin: padding literals are always FALSE
        g.sync();  // the scatter above wrote rows that other threads own in the stage loops

        // The step size after an accepted step (CpuRungeKutta.cpp:252-256) is needed only
        // from the next step's stage 2 on, so it is formed during the next stage 1, after
        // the clause loop, by lane 0 of the last warp: that warp has no more clauses than
        // the first, so the FP64 pow() runs while the first warps finish theirs.
        double hnext = 1e-9, e_acc = 0.0, h_acc = 0.0;
        bool h_pending = false;
        const int pow_tid = nt >= 64 ? nt - 32 : 0;
        auto settle_h = [&]() {
            if (h_pending && tid == pow_tid)
                red_d[34] = e_acc > ck::ERRCON ? __dmul_rn(__dmul_rn(ck::SAFETY, h_acc), pow(e_acc, ck::PGROW))
                                               : __dmul_rn(5.0, h_acc);
        };
        auto take_h = [&]() {
            if (h_pending) hnext = red_d[34];
            h_pending = false;
        };

        // One RHS evaluation at stage S; the derivative lands in slot S of the rows, or
        // for S == 6 is consumed at once into the candidate state (slot 2) and the error
        // norm.  The spins' stage input is formed by the variable phase of the stage
        // before (ready = true; stage 1's by the accepted step's copy), or here.
        auto eval = [&](auto stage, float hT, float h0T, float& em, bool ready) {
            constexpr int S = decltype(stage)::value;
            if (!ready)
                for (int v = tid; v < n; v += nt)
                    put_spin(v, row_input<S>(load_row<S, R>(rs.at(v)), hT));
            g.sync();
            if constexpr (ROWS_G) {
                const int np = I.nparts, ns1 = ((n + 31) >> 5) + 1;
                for (int pp = 0; pp < np; pp++) {
                    const int c0 = ld_ro(I.part_c0 + pp), c1 = ld_ro(I.part_c0 + pp + 1);
                    const uint32_t* lp = I.plit + lean_word_index(c0 + tid, 0, K);
                    typename R::Ref ra = rs.at(cb + c0 + tid);
                    for (int c = c0 + tid; c < c1; c += nt, lp += (size_t)nt * K, ra = R::advance(ra, nt)) {
                        const Row6 o = load_clause_row<S, R>(ra, ready);
                        const float d = part_clause<K>(sb, cs0, lp, exp2_fast(row_input<S>(o, hT)) * a2n, duc);
                        if constexpr (S < 6) {
                            R::st(ra, S, d);
                        } else {
                            em = fmaxf(em, rk_err_ratio(o.x, o.k1, o.k3, o.k4, o.k5, d, hT, h0T, true));
                            R::st(ra, 2, rk_new<float>(o.x, o.k1, o.k3, o.k4, d, hT));
                        }
                    }
                    if constexpr (S == 1)
                        if (pp + 1 == np) settle_h();
                    g.sync();
                    if constexpr (S == 1)
                        if (pp + 1 == np) take_h();
                    // each variable's sum continues from the previous part (kept in slot S,
                    // or for S = 6 in slot 2, whose K2 the stage-6 input has read already)
                    constexpr int SLOT = S < 6 ? S : 2;
                    const bool last = pp + 1 == np;
                    // What a variable needs from L2 (occurrence count, SELL row, its row for
                    // the next stage's input or stage 6, the sum so far), then its sum over
                    // the part's slots; two variables at a time, both loaded first, so the
                    // L2 latencies overlap.
                    struct VarIn {
                        int cnt, r0;
                        float sum;
                        Row6 o;
                    };
                    auto var_load = [&](int v) {
                        VarIn a;
                        a.cnt = (int)I.part_cnt[(size_t)pp * n + v];
                        a.r0 = ld_ro(I.part_srow + (size_t)pp * ns1 + (v >> 5));
                        const typename R::Ref r = rs.at(v);
                        if (last) a.o = load_row<S, R>(r);
                        a.sum = pp == 0 ? 0.0f : R::ld(r, SLOT);
                        return a;
                    };
                    auto var_sum = [&](int v, const VarIn& a) {
                        uint32_t pa = cs0 + 4u * (uint32_t)(a.r0 * 32 + (v & 31));
                        float sum = a.sum;
#pragma unroll 8
                        for (int k = 0; k < a.cnt; k++, pa += 128u) sum = sum + lds(pa);
                        const typename R::Ref r = rs.at(v);
                        if (!last) {
                            R::st(r, SLOT, sum);
                        } else if constexpr (S < 6) {
                            Row6 o = a.o;
                            R::st(r, S, sum);
                            set_k<S>(o, sum);
                            put_spin(v, row_input<S + 1>(o, S == 1 ? (float)hnext : hT));
                        } else {
                            const Row6& o = a.o;
                            em = fmaxf(em, rk_err_ratio(o.x, o.k1, o.k3, o.k4, o.k5, sum, hT, h0T, false));
                            R::st(r, 2, rk_new<float>(o.x, o.k1, o.k3, o.k4, sum, hT));
                        }
                    };
                    for (int v = tid; v < n; v += 2 * nt) {
                        const bool two = v + nt < n;
                        const VarIn a = var_load(v);
                        VarIn b2;
                        if (two) b2 = var_load(v + nt);
                        var_sum(v, a);
                        if (two) var_sum(v + nt, b2);
                    }
                    if (!last) g.sync();  // the next part's clauses reuse the slots
                }
                return;
            }
            const uint32_t* lp = I.flit + lean_word_index(tid, 0, K);
            typename R::Ref ra = rs.at(cb + tid);
            for (int c = tid; c < m; c += nt, lp += (size_t)nt * K, ra = R::advance(ra, nt)) {
                const Row6 o = load_clause_row<S, R>(ra, ready);
                const float d = fast_clause<K>(sb, mask, cs0, lp, exp2_fast(row_input<S>(o, hT)) * a2n, duc);
                if constexpr (S < 6) {
                    R::st(ra, S, d);
                } else {
                    em = fmaxf(em, rk_err_ratio(o.x, o.k1, o.k3, o.k4, o.k5, d, hT, h0T, true));
                    R::st(ra, 2, rk_new<float>(o.x, o.k1, o.k3, o.k4, d, hT));
                }
            }
            if constexpr (S == 1) settle_h();
            g.sync();
            if constexpr (S == 1) take_h();
            for (int v = tid; v < n; v += nt) {
                const int g32 = v >> 5;
                const int r0 = ld_ro(I.srow + g32), r1 = ld_ro(I.srow + g32 + 1);
                uint32_t p = cs0 + 4u * (uint32_t)(r0 * 32 + (v & 31));
                const typename R::Ref r = rs.at(v);
                Row6 o = load_row<S, R>(r);  // what the next stage's input (or stage 6) reads
                float sum = 0.0f;
#pragma unroll 8
                for (int k = r0; k < r1; k++, p += 128u) sum = sum + lds(p);
                if constexpr (S < 6) {
                    R::st(r, S, sum);
                    set_k<S>(o, sum);
                    put_spin(v, row_input<S + 1>(o, S == 1 ? (float)hnext : hT));
                } else {
                    em = fmaxf(em, rk_err_ratio(o.x, o.k1, o.k3, o.k4, o.k5, sum, hT, h0T, false));
                    R::st(r, 2, rk_new<float>(o.x, o.k1, o.k3, o.k4, sum, hT));
                }
            }
        };

        double t = 0.0, hdid = 0.0;
        // after an accepted step: the spins hold its state (stage 1's input) and the clause
        // rows' state is still in slot 2 until the next stage 1 moves it
        bool s1_ready = false;
        int steps = 0, attempts = 0, rhs = 0, viol = -1, minviol = INT_MAX;
        int status = SAT_UNKNOWN;

        while (status == SAT_UNKNOWN && t < P.tmax && steps < P.maxsteps) {
            bool underflow = false, interrupted = false;
            int taken = 0;
            for (int b = 0; b < P.batch; b++) {
                float dummy = 0.0f;
                eval(std::integral_constant<int, 1>{}, 0.0f, 0.0f, dummy, s1_ready);
                s1_ready = false;  // the clause rows' copy is done
                rhs++;
                const double h0 = hnext;
                const float h0T = (float)h0;
                double h = hnext, ermax = 0.0;
                bool retry = false;  // a retry's stage-2 input uses the smaller step
                while (true) {
                    const float hT = (float)h;
                    float em = 0.0f;
                    eval(std::integral_constant<int, 2>{}, hT, h0T, em, !retry);
                    eval(std::integral_constant<int, 3>{}, hT, h0T, em, true);
                    eval(std::integral_constant<int, 4>{}, hT, h0T, em, true);
                    eval(std::integral_constant<int, 5>{}, hT, h0T, em, true);
                    // another start's solution (stop-on-first), read now so that the read
                    // completes during stage 6
                    int other_solved = 0;
                    if (tid == 0 && P.stop_on_first) other_solved = ld_relaxed(P.inst_solved + pidx);
                    eval(std::integral_constant<int, 6>{}, hT, h0T, em, true);
                    rhs += 5;
                    attempts++;
                    ermax = lean_max_then(em, red_u, red_d, [&](double emax) {
                        const double e = __ddiv_rn(emax, P.eps);
                        if (e > 1.0)  // rejected: the retry's step size now (accepted: settle_h)
                            red_d[34] = fmax(__dmul_rn(__dmul_rn(ck::SAFETY, h), pow(e, ck::PSHRNK)),
                                             __dmul_rn(ck::HFACTOR, h));
                        const bool quit = other_solved != 0 || (P.deadline && globaltimer_ns() >= deadline);
                        red_d[35] = quit ? 1.0 : 0.0;
                        return e;
                    });
                    if (red_d[35] != 0.0) { interrupted = true; break; }
                    if (ermax <= 1.0) {
                        e_acc = ermax;
                        h_acc = h;
                        h_pending = true;
                        break;
                    }
                    h = red_d[34];
                    retry = true;
                    if (__dadd_rn(t, h) == t) { underflow = true; break; }
                }
                if (underflow || interrupted) break;
                hdid = h;
                t = __dadd_rn(t, h);
                taken++;
                // accept: the candidate state (slot 2) becomes the state, each element by
                // the thread that owns it in the stage loops; the spins are also the next
                // stage 1's input.  The clause rows follow in that stage's clause loop.
                for (int v = tid; v < n; v += nt) {
                    const typename R::Ref r = rs.at(v);
                    const float xn = R::ld(r, 2);
                    R::st(r, 0, xn);
                    put_spin(v, xn);
                }
                s1_ready = true;
            }
            if (underflow) { status = SAT_UNDERFLOW; break; }
            steps += taken;
            if (interrupted) { status = SAT_ODE_INTERRUPTED; break; }

            // CpuSat::GetClauseViolationCount on the accepted state
            for (int v = tid; v < n; v += nt) sts(sb + 4u * (uint32_t)v, R::ld(rs.at(v), 0));
            g.sync();
            int cnt = 0;
            {
                const uint32_t* lp = (ROWS_G ? I.plit : I.flit) + lean_word_index(tid, 0, K);
                for (int c = tid; c < m; c += nt, lp += (size_t)nt * K) {
                    bool sat = false;
#pragma unroll
                    for (int q = 0; q < K; q++) {
                        const uint32_t w = ld_lit(lp + 32 * q);
                        // the positive spin (the word of a negated literal points at -s)
                        const uint32_t sa = ROWS_G ? sb + 4u * (w & 0x1FFFu)
                                                   : (w & 0x80000000u) ? (sb | (w & mask)) - 4u * (uint32_t)neg_spin_base(n)
                                                                       : (sb | (w & mask));
                        const bool tv = lds(sa) > 0.0f;
                        sat |= (w & 0x80000000u) ? !tv : tv;
                    }
                    cnt += sat ? 0 : 1;
                }
            }
            viol = group_sum<1>(g, cnt, red_i);
            if (viol < minviol) {
                minviol = viol;
                if (P.best_bits) {
                    uint32_t* bits = P.best_bits + P.unit_bits[u];
                    for (int i0 = tid & ~31; i0 < n; i0 += nt) {
                        const int i = i0 + (tid & 31);
                        const bool bb = i < n && sy[__ldg(I.iperm + (i < n ? i : 0))] > 0.0f;
                        const unsigned bal = __ballot_sync(0xffffffffu, bb);
                        if ((tid & 31) == 0) bits[i0 >> 5] = bal;
                    }
                }
            }
            if (viol == 0) {
                status = SAT_SOLUTION_FOUND;
                if (tid == 0 && P.stop_on_first) atomicExch(P.inst_solved + pidx, 1);
                break;
            }
            int f = 0;
            if (tid == 0) {
                if (P.deadline && globaltimer_ns() >= *P.deadline) f = 1;
                if (P.stop_on_first && atomicAdd(P.inst_solved + pidx, 0) != 0) f = 1;
            }
            if (g.bcast(&s_flag, f)) { status = SAT_ODE_INTERRUPTED; break; }
        }
        if (status == SAT_UNKNOWN) {
            if (t >= P.tmax) status = SAT_MAXTIME_REACHED;
            else if (steps >= P.maxsteps) status = SAT_MAXITER_REACHED;
        }

        // write back the final state in the public layout
        g.sync();
        for (int i = tid; i < n; i += nt) G[i] = R::ld(rs.at(__ldg(I.iperm + i)), 0);
        for (int j = tid; j < m; j += nt) G[n + j] = exp2f(R::ld(rs.at(cb + __ldg(icp + j)), s1_ready ? 2 : 0));
        if (tid == 0) {
            UnitResult r;
            r.time = t; r.hdid = hdid; r.status = status; r.steps = steps; r.attempts = attempts;
            r.rhs = rhs; r.viol = viol; r.min_viol = minviol == INT_MAX ? -1 : minviol;
            r.pad0 = r.pad1 = 0;
            P.results[u] = r;
        }
        g.sync();
    }
}

}  // namespace asb
