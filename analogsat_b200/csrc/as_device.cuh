// Device-side building blocks of the AnalogSAT CTDS hot path on sm_100a.
//
// The ODE (AnalogSAT/cpu_sat/CpuSat.cpp:199-241, cpu_helper.h:101-126):
//   K_m    = 2^-K prod_q (1 - c_mq s_q)            (K = max clause length)
//   ds_i   = sum_m 2 a_m c_mi K_mi K_m,  K_mi = 2^-K prod_{q != i} (1 - c_mq s_q)
//   da_m   = a_m K_m^2   (FP32 path: a_m is held as u_m = log2 a_m, du_m = K_m^2 / ln 2)
//
// One RHS evaluation is two block-wide phases over shared memory:
//   clause phase  thread-per-clause: gather K spins from `sy`, form K_m and the
//                 leave-one-out products in registers, store each literal's
//                 contribution 2 c K_mi K_m a_m straight into its variable's slot of
//                 the SELL-32 contribution buffer `cs`, return da_m;
//   var phase     thread-per-variable: sum the variable's row of `cs` (contiguous,
//                 bank-conflict free, no index loads) in clause order.
// No atomics anywhere, so results are deterministic; in FP64 every operation is
// an explicitly rounded mul/add in the reference's order, which makes the RHS
// bit-identical to CpuSat<double>.  Layouts are documented in as_problem.h.
#pragma once

#include <cooperative_groups.h>
#include <cstdint>
#include <cuda_runtime.h>

namespace asb {

// One packed instance in device memory.
struct DevInstance {
    int n, m, k, mp, nslices, nslots;
    const uint32_t* lit;    // [k][mp] compact literal words (var | sign | slot), or null
    const uint32_t* litw;   // [k][mp] wide literal words: sign << 31 | variable
    const uint32_t* slotw;  // [k][mp] contribution slot of each wide literal
    const int32_t* srow;   // [nslices + 1] SELL row offsets
    const int32_t* perm;    // internal -> public variable
    const int32_t* iperm;   // public -> internal variable
    const int32_t* icperm;  // public -> internal clause
    const int32_t* cperm;   // internal -> public clause
    // CTDS variant (the reference's ISat implementations): tanh = 0 CpuSat / CudaSat,
    // tanh = 1 CpuSatTanh / CudaSatTanh with slope q; bias b (ISat::Set_B) adds
    // mean(a) (M/N) b knorm^2 (pi/2) sin(pi s_i) to ds_i (0: off).
    int tanh;
    double q, b;
    // Lean FP32 solver layout (solve_kernel_fast), or null when the instance does not
    // qualify: literal words flit[lean_word_index(m, q, k)] (blocked by 32 clauses,
    // as_fast.cuh) that carry shared-memory addressing -- bit 31 negated literal, bits
    // 14-30 the literal's contribution slot, bits 0-13 the byte offset of its spin (the
    // spins sit at the spin base, spin_align-aligned, the slots at cs_off from it, the
    // interleaved RK stage rows at rows_off or, blocked, in a global slab).
    const uint32_t* flit;
    int cs_off, rows_off, cs_off_g;  // cs_off_g: the global-rows form's slots (one spin copy)
    // Clause parts of the lean kernel's global-rows form (PartLayout in as_problem.h):
    // words plit[lean_word_index(m, q, k)] = sign | slot in the part's buffer << 13 |
    // internal variable, part p's internal clauses [part_c0[p], part_c0[p + 1]), SELL
    // rows part_srow[p * (nslices + 1) + g], occurrences part_cnt[p * n + v], its own
    // clause order picperm (public -> internal); nparts = 0 when the instance has no
    // such layout.
    const uint32_t* plit;
    const int32_t* part_c0;
    const int32_t* part_srow;
    const uint16_t* part_cnt;
    const int32_t* picperm;
    int nparts, part_slots;
};

constexpr float kInvLn2 = 1.4426950408889634f;  // d(log2 a)/dt = (da/dt) / (a ln 2)

// ---- explicitly rounded arithmetic: FP64 follows the reference bit for bit ----
template <typename T> struct Arith;
template <> struct Arith<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};
template <> struct Arith<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
};

// The bias term is on: CpuSat adds it when b knorm^2 > 0 (CpuSat.cpp:229), CpuSatTanh
// always (CpuSatTanh.cpp:233-238, where b = 0 adds zeros).
__device__ __forceinline__ bool bias_on(const DevInstance& I) { return I.b > 0.0 || I.tanh; }

// mean(a) (M/N) b knorm^2 (pi/2): the per-call factor of the bias term, formed in the
// reference's expression order from the clause-weight sum (CpuSat.cpp:230-236).
template <typename T>
__device__ __forceinline__ T bias_factor(const DevInstance& I, double asum, T knorm) {
    using A = Arith<T>;
    const T a = (T)asum / (T)I.m;
    const T alpha = (T)I.m / (T)I.n;
    const T bb = A::mul(A::mul((T)I.b, knorm), knorm);
    return A::mul(A::mul(A::mul(a, alpha), bb), T(1.570796326794897));
}
// ... times sin(pi s_i) added to the variable's sum
__device__ __forceinline__ double bias_term(double f, double s) { return __dmul_rn(f, sin(__dmul_rn(s, 3.141592653589793))); }
__device__ __forceinline__ float bias_term(float f, float s) { return f * sinf(s * 3.14159265f); }
__device__ __forceinline__ double tanh_t(double x) { return tanh(x); }
__device__ __forceinline__ float tanh_t(float x) { return tanhf(x); }

// 2^u with the SFU (relative error ~2^-22, below the FP32 state's own rounding)
__device__ __forceinline__ float exp2_fast(float u) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(u));
    return r;
}


// Read-only loads of instance data, kept inside the stage loop (hoisting them would
// cost registers across all six stages; they hit L1).
__device__ __forceinline__ uint32_t ld_ro(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::evict_last.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ int32_t ld_ro(const int32_t* p) {
    int32_t v;
    asm volatile("ld.global.nc.L1::evict_last.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// One literal of a clause.  ENC 0: compact word (sign | 15-bit variable | 16-bit
// slot), one load.  ENC 1: wide words (sign | 31-bit variable, 32-bit slot), two loads,
// for instances beyond the compact limits.
template <int ENC> struct Lit;
template <> struct Lit<0> {
    uint32_t w;
    __device__ __forceinline__ void load(const DevInstance& I, int idx) { w = ld_ro(I.lit + idx); }
    __device__ __forceinline__ uint32_t var() const { return (w >> 16) & 0x7fffu; }
    __device__ __forceinline__ uint32_t slot() const { return w & 0xffffu; }
    __device__ __forceinline__ bool neg() const { return (w >> 31) != 0; }
};
template <> struct Lit<1> {
    uint32_t w, s;
    __device__ __forceinline__ void load(const DevInstance& I, int idx) {
        w = ld_ro(I.litw + idx);
        s = ld_ro(I.slotw + idx);
    }
    __device__ __forceinline__ uint32_t var() const { return w & 0x7fffffffu; }
    __device__ __forceinline__ uint32_t slot() const { return s; }
    __device__ __forceinline__ bool neg() const { return (w >> 31) != 0; }
};

// Clause phase for one clause m: stores the per-literal spin contributions into cs
// and returns da_m (du_m in log space).  `am` is a_m in linear space.
// EXACT: every clause has exactly KMAX slots (shorter clauses are padded with the
// sentinel word, whose contribution goes to the trash slot), so no runtime length
// tests are needed; otherwise the runtime length k <= KMAX is honoured.  For
// k <= 10 the leave-one-out products follow CpuProdWrapper (ascending,
// left-associated); for k > 10 the generic CalculateAll form (CpuSat.cpp:291-349).
template <typename T, bool LOGA, int KMAX, bool EXACT, int ENC>
__device__ __forceinline__ T clause_phase(const DevInstance& I, int m, const T* __restrict__ sy,
                                          T* __restrict__ cs, T am, T knorm) {
    using A = Arith<T>;
    // FP32 with log-space weights folds the power-of-two scalings (knorm = 2^-k): km
    // holds P = f_0 .. f_{k-1} (K_m = knorm P), and 2 r = P (a_m 2 knorm^2), du_m =
    // (P P)(knorm^2 / ln 2) -- the same roundings as the unfolded forms, since a
    // power-of-two factor scales a rounded product exactly (the lean kernel forms them so)
    constexpr bool kFold = LOGA && sizeof(T) == 4;
    Lit<ENC> w[KMAX];
    T f[KMAX];
    T km = knorm;
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (EXACT || q < I.k) {
            w[q].load(I, q * I.mp + m);
            const T s = sy[w[q].var()];
            if constexpr (sizeof(T) == 4)  // 1 - (-s) == 1 + s: the literal's sign bit flips s
                f[q] = T(1) - __int_as_float(__float_as_int(s) ^ (int)(w[q].w & 0x80000000u));
            else
                f[q] = w[q].neg() ? A::add(T(1), s) : A::sub(T(1), s);
            km = (kFold && q == 0) ? f[q] : A::mul(km, f[q]);
        }
    }
    T dam;
    if constexpr (kFold) dam = (km * km) * (knorm * knorm * T(kInvLn2));
    else if constexpr (LOGA) dam = km * km * T(kInvLn2);
    else dam = A::mul(A::mul(am, km), km);
    if (I.tanh) {
        // CpuSatTanh: knorm a_m |K_mi| tanh(q (1 - c s_i)) c_mi (KmiFuncTanh,
        // cpu_helper.h:115-125, leave-one-out product as CpuProdWrapper; k > 10: the
        // generic CalculateAll, CpuSatTanh.cpp:250-297)
        const T q = (T)I.q;
        if (KMAX <= 10 || I.k <= 10) {
            const T r = A::mul(knorm, am);
#pragma unroll
            for (int qq = 0; qq < KMAX; qq++) {
                if (EXACT || qq < I.k) {
                    T prod = T(1);
                    bool first = true;
#pragma unroll
                    for (int l = 0; l < KMAX; l++) {
                        if (l != qq && (EXACT || l < I.k)) {
                            prod = first ? f[l] : A::mul(prod, f[l]);
                            first = false;
                        }
                    }
                    const T rr = A::mul(A::mul(r, fabs(prod)), tanh_t(A::mul(q, f[qq])));
                    cs[w[qq].slot()] = w[qq].neg() ? -rr : rr;
                }
            }
        } else {
#pragma unroll
            for (int qq = 0; qq < KMAX; qq++) {
                if (EXACT || qq < I.k) {
                    T temp = T(1);
#pragma unroll
                    for (int l = 0; l < KMAX; l++)
                        if (EXACT || l < I.k) temp = A::mul(temp, l == qq ? T(1) : f[l]);
                    T rr = A::mul(A::mul(knorm, am), fabs(temp));
                    rr = w[qq].neg() ? -rr : rr;
                    cs[w[qq].slot()] = A::mul(rr, tanh_t(A::mul(q, f[qq])));
                }
            }
        }
        return dam;
    }
    if (KMAX <= 10 || I.k <= 10) {
        // r (r2 = 2 r when folded)
        const T r = kFold ? km * (am * (T(2) * knorm * knorm)) : A::mul(A::mul(km, knorm), am);
#pragma unroll
        for (int q = 0; q < KMAX; q++) {
            if (EXACT || q < I.k) {
                T prod = T(1);
                bool first = true;
#pragma unroll
                for (int l = 0; l < KMAX; l++) {
                    if (l != q && (EXACT || l < I.k)) {
                        prod = first ? f[l] : A::mul(prod, f[l]);
                        first = false;
                    }
                }
                if constexpr (sizeof(T) == 4) {  // (2r) prod == 2 (r prod) above the subnormals
                    const T rr = (kFold ? r : r + r) * prod;
                    cs[w[q].slot()] = __int_as_float(__float_as_int(rr) ^ (int)(w[q].w & 0x80000000u));
                } else {
                    T rr = A::mul(r, prod);
                    rr = rr + rr;
                    cs[w[q].slot()] = w[q].neg() ? -rr : rr;
                }
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < KMAX; q++) {
            if (EXACT || q < I.k) {
                T temp = kFold ? knorm * km : km;
#pragma unroll
                for (int l = 0; l < KMAX; l++)
                    if (EXACT || l < I.k) temp = A::mul(temp, l == q ? T(1) : f[l]);
                const T rr = A::mul(A::mul(A::mul(T(2), temp), knorm), am);
                cs[w[q].slot()] = w[q].neg() ? -rr : rr;
            }
        }
    }
    return dam;
}

// Var phase for internal variable v (< n): sum of its SELL row in clause order.
// Padding slots are zero (x + 0 == x, and the reference's sums are never -0).
template <typename T>
__device__ __forceinline__ T var_phase(const DevInstance& I, int v, const T* __restrict__ cs) {
    using A = Arith<T>;
    const int g = v >> 5;
    const int r0 = ld_ro(I.srow + g), r1 = ld_ro(I.srow + g + 1);
    const T* p = cs + r0 * 32 + (v & 31);
    T sum = T(0);
#pragma unroll 4
    for (int r = r0; r < r1; r++, p += 32) sum = A::add(sum, *p);
    return sum;
}

// Clause check for clause m against the spins in sy (CpuSat.cpp:136-164): a
// variable is TRUE when s > 0; the sentinel (s = -1, positive) is FALSE.
template <int KMAX, bool EXACT, int ENC, typename T>
__device__ __forceinline__ int clause_violated(const DevInstance& I, int m, const T* sy) {
    bool sat = false;
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (EXACT || q < I.k) {
            Lit<ENC> w;
            w.load(I, q * I.mp + m);
            const bool t = sy[w.var()] > T(0);
            sat |= w.neg() ? !t : t;
        }
    }
    return sat ? 0 : 1;
}

// ---- block reductions (warp shuffles + one smem slot per warp) ----
// red holds one slot per warp of the launch (blockDim.x / 32 <= 32).
__device__ __forceinline__ int block_sum(int v, int* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();  // red may still be read from the previous reduction
    if (lane == 0) red[warp] = v;
    __syncthreads();
    int s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    return s;
}

// ---- thread groups: one CTA, or a thread-block cluster of CL CTAs cooperating on one
// trajectory (global-storage mode).  Group-wide barriers are __syncthreads or the
// cluster barrier (release/acquire at cluster scope, which orders the global-memory
// slab accesses of all CTAs); values decided by one thread are published to every
// CTA's shared memory through distributed shared memory.
template <int CL>
struct Grp {
    int rank, gtid, gnt;
    __device__ __forceinline__ Grp() {
        if constexpr (CL == 1) {
            rank = 0;
        } else {
            rank = (int)cooperative_groups::this_cluster().block_rank();
        }
        gtid = rank * (int)blockDim.x + (int)threadIdx.x;
        gnt = CL * (int)blockDim.x;
    }
    __device__ __forceinline__ void sync() const {
        if constexpr (CL == 1) __syncthreads();
        else cooperative_groups::this_cluster().sync();
    }
    // Group thread 0 publishes v into `slot` (a __shared__ variable) of every CTA.
    template <typename V>
    __device__ __forceinline__ V bcast(V* slot, V v) const {
        if (gtid == 0) {
            if constexpr (CL == 1) {
                *slot = v;
            } else {
                auto cl = cooperative_groups::this_cluster();
                for (int r = 0; r < CL; r++) *cl.map_shared_rank(slot, r) = v;
            }
        }
        sync();
        return *slot;
    }
};

// Group-wide max (FP64) post-processed by one thread: fn(max) is broadcast to every
// thread.  red: 36 doubles of shared memory per CTA -- [0,32) warp partials, [32] the
// CTA partial, [33] the result; fn may publish more values in red[34] and red[35].
template <int CL, typename F>
__device__ __forceinline__ double group_max_then(const Grp<CL>& g, double v, double* red, F&& fn) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();  // red may still be read from the previous reduction
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
        red[32] = m;
    }
    if constexpr (CL > 1) {
        g.sync();
        if (threadIdx.x == 0) {
            auto cl = cooperative_groups::this_cluster();
            double m = red[32];
            for (int r = 0; r < CL; r++) m = fmax(m, *cl.map_shared_rank(red + 32, r));
            red[33] = fn(m);
        }
    } else {
        if (threadIdx.x == 0) red[33] = fn(red[32]);
    }
    __syncthreads();
    return red[33];
}

// Group-wide integer sum (red: 33 ints per CTA).
template <int CL>
__device__ __forceinline__ int group_sum(const Grp<CL>& g, int v, int* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    int s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    if constexpr (CL > 1) {
        if (threadIdx.x == 0) red[32] = s;
        g.sync();
        auto cl = cooperative_groups::this_cluster();
        s = 0;
        for (int r = 0; r < CL; r++) s += *cl.map_shared_rank(red + 32, r);
        g.sync();  // red[32] of every CTA may be rewritten after this point
    }
    return s;
}

// Block max (FP64) whose result is post-processed by thread 0 (single-CTA kernels).
template <typename F>
__device__ __forceinline__ double block_max_then(double v, double* red, F&& fn) {
    return group_max_then<1>(Grp<1>(), v, red, fn);
}

}  // namespace asb
