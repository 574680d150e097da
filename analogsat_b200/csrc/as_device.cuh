// Device-side building blocks of the AnalogSAT CTDS hot path on sm_100a.
//
// The ODE (AnalogSAT/cpu_sat/CpuSat.cpp:199-241, cpu_helper.h:101-126):
//   K_m    = 2^-K prod_q (1 - c_mq s_q)            (K = max clause length)
//   ds_i   = sum_m 2 a_m c_mi K_mi K_m,  K_mi = 2^-K prod_{q != i} (1 - c_mq s_q)
//   da_m   = a_m K_m^2        (log space: du_m = K_m^2 with u_m = ln a_m)
//
// One RHS evaluation is two block-wide phases over shared memory:
//   clause phase  thread-per-clause: gather K spins from `sy`, form K_m and the
//                 leave-one-out products in registers, write each literal's
//                 contribution 2 c K_mi K_m a_m to `contrib[q*mp + m]`
//                 (coalesced, conflict-free) and return da_m;
//   var phase     thread-per-variable: walk the variable's SELL-32 row list
//                 (coalesced loads) and sum its contributions in clause order.
// No atomics anywhere, so results are deterministic; in FP64 every operation is
// an explicitly rounded mul/add in the reference's order, which makes the RHS
// bit-identical to CpuSat<double>.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace asb {

// One packed instance in device memory (layout documented in as_problem.h).
struct DevInstance {
    int n, m, k, mp, nslices, pad;
    const uint32_t* lit;
    const int32_t* sell_row;
    const int32_t* sell;
};

// ---- explicitly rounded arithmetic: FP64 follows the reference bit for bit ----
template <typename T> struct Arith;
template <> struct Arith<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double ex(double u) { return exp(u); }
    static __device__ __forceinline__ double lg(double a) { return log(a); }
};
template <> struct Arith<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float ex(float u) { return expf(u); }
    static __device__ __forceinline__ float lg(float a) { return logf(a); }
};

__device__ __forceinline__ uint32_t lit_var(uint32_t w) { return w & 0x7fffffffu; }

// Read-only loads of instance data that the compiler must not hoist out of the RK
// stage loop (keeping them live across stages would cost registers, not traffic:
// they hit L1).
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
__device__ __forceinline__ bool lit_neg(uint32_t w) { return (w >> 31) != 0; }

// Clause phase for one clause m: returns da_m (or du_m in log space), writes the
// per-literal spin contributions into contrib.  `am` is a_m in linear space.
// KMAX bounds the runtime clause length k.  For k <= 10 the leave-one-out
// products follow CpuProdWrapper (ascending, left-associated); for k > 10 the
// generic CalculateAll form (CpuSat.cpp:291-349) is used.
template <typename T, bool LOGA, int KMAX>
__device__ __forceinline__ T clause_phase(const DevInstance& I, int m, const T* __restrict__ sy,
                                          T* __restrict__ contrib, T am, T knorm) {
    using A = Arith<T>;
    uint32_t w[KMAX];
    T f[KMAX];
    T km = knorm;
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (q < I.k) {
            w[q] = ld_ro(I.lit + (size_t)q * I.mp + m);
            const T s = sy[lit_var(w[q])];
            f[q] = lit_neg(w[q]) ? A::add(T(1), s) : A::sub(T(1), s);
            km = A::mul(km, f[q]);
        }
    }
    const T dam = LOGA ? A::mul(km, km) : A::mul(A::mul(am, km), km);
    if (KMAX <= 10 || I.k <= 10) {
        const T r = A::mul(A::mul(km, knorm), am);
#pragma unroll
        for (int q = 0; q < KMAX; q++) {
            if (q < I.k && lit_var(w[q]) != (uint32_t)I.n) {
                T prod = T(1);
                bool first = true;
#pragma unroll
                for (int l = 0; l < KMAX; l++) {
                    if (l != q && l < I.k) {
                        prod = first ? f[l] : A::mul(prod, f[l]);
                        first = false;
                    }
                }
                T rr = A::mul(r, prod);
                rr = lit_neg(w[q]) ? -(rr + rr) : (rr + rr);
                contrib[q * I.mp + m] = rr;
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < KMAX; q++) {
            if (q < I.k && lit_var(w[q]) != (uint32_t)I.n) {
                T temp = km;
#pragma unroll
                for (int l = 0; l < KMAX; l++)
                    if (l < I.k) temp = A::mul(temp, l == q ? T(1) : f[l]);
                T rr = A::mul(A::mul(A::mul(T(2), temp), knorm), am);
                contrib[q * I.mp + m] = lit_neg(w[q]) ? -rr : rr;
            }
        }
    }
    return dam;
}

// Var phase for variable i (< n): sum of its contributions in (clause, slot) order.
template <typename T>
__device__ __forceinline__ T var_phase(const DevInstance& I, int i, const T* __restrict__ contrib) {
    using A = Arith<T>;
    const int g = i >> 5, lane = i & 31;
    const int r0 = ld_ro(I.sell_row + g), r1 = ld_ro(I.sell_row + g + 1);
    T sum = T(0);
    for (int r = r0; r < r1; r++) {
        const int e = ld_ro(I.sell + (size_t)r * 32 + lane);
        if (e < 0) break;
        sum = A::add(sum, contrib[e]);
    }
    return sum;
}

// Clause check for clause m against the spins in sy (CpuSat.cpp:136-164): a
// variable is TRUE when s > 0; the sentinel (s = -1, positive) is FALSE.
template <int KMAX>
__device__ __forceinline__ int clause_violated(const DevInstance& I, int m, const float* sy) {
    bool sat = false;
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (q < I.k) {
            const uint32_t w = __ldg(I.lit + (size_t)q * I.mp + m);
            const bool t = sy[lit_var(w)] > 0.0f;
            sat |= lit_neg(w) ? !t : t;
        }
    }
    return sat ? 0 : 1;
}

template <int KMAX>
__device__ __forceinline__ int clause_violated(const DevInstance& I, int m, const double* sy) {
    bool sat = false;
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (q < I.k) {
            const uint32_t w = __ldg(I.lit + (size_t)q * I.mp + m);
            const bool t = sy[lit_var(w)] > 0.0;
            sat |= lit_neg(w) ? !t : t;
        }
    }
    return sat ? 0 : 1;
}

// ---- block reductions (warp shuffles + one smem slot per warp) ----
template <int BT>
__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();  // red may still be read from the previous reduction
    if (lane == 0) red[warp] = v;
    __syncthreads();
    v = red[0];
#pragma unroll
    for (int w = 1; w < BT / 32; w++) v = fmax(v, red[w]);
    return v;
}

template <int BT>
__device__ __forceinline__ int block_sum(int v, int* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    int s = 0;
#pragma unroll
    for (int w = 0; w < BT / 32; w++) s += red[w];
    return s;
}

}  // namespace asb
