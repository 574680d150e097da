// Kernels of the AnalogSAT B200 hot path.
//
//  solve_kernel    persistent RK45 (Cash-Karp) integrator: one CTA per trajectory,
//                  work units popped from a global counter (dynamic refill); the
//                  whole trajectory -- RK stage vectors, spins, clause contributions
//                  -- lives in shared memory for its lifetime; batched clause check
//                  and early exit on device.  Replaces SatSolver::DoSolve + CpuRungeKutta::Step/rkqs/
//                  rkck + CpuSat::GetDerivatives/GetClauseViolationCount
//                  (AnalogSAT/solver/SatSolver.h:273-355,
//                  AnalogSAT/cpu_sat/CpuRungeKutta.cpp:66-100,181-267,
//                  AnalogSAT/cpu_sat/CpuSat.cpp:65-94,136-173,199-241).
//  rhs_batch_kernel   standalone RHS over many trajectories whose state lives in
//                  HBM (ISat::GetDerivatives, AnalogSAT/solver/IODE.h).
//  viol_batch_kernel  exact unsat counts for many states (ISat::GetClauseViolationCount).
#pragma once

#include <climits>
#include "as_device.cuh"

namespace asb {

enum : int {
    SAT_SOLUTION_FOUND = 0,
    SAT_UNDERFLOW = 1,
    SAT_ODE_INTERRUPTED = 2,
    SAT_MAXTIME_REACHED = 3,
    SAT_MAXITER_REACHED = 4,
    SAT_UNKNOWN = 5,
};

struct UnitResult {
    double time;      // integrated analog time
    double hdid;      // last accepted step size
    int status;       // SatResult code
    int steps;        // accepted steps (SatSolver counting: whole batches)
    int attempts;     // attempted steps incl. rejections
    int rhs;          // RHS evaluations
    int viol;         // unsat count at the last check
    int min_viol;     // smallest unsat count seen at any check
    int pad0, pad1;
};

struct SolveParams {
    const DevInstance* inst;     // [num_instances]
    const int* unit_inst;        // [num_units]
    const long long* unit_state; // [num_units] element offset of the unit's public state
    void* states;                // public layout [s_1..s_N, a_1..a_M] per unit (T)
    UnitResult* results;         // [num_units]
    int* queue_head;             // work counter, zero before launch
    int* inst_solved;            // [num_instances] first-solution flags
    uint32_t* best_bits;         // optional: per unit ceil(N/32) words, assignment at min_viol
    const long long* unit_bits;  // [num_units] word offset into best_bits
    int num_units;
    int maxsteps;
    int batch;
    int stop_on_first;           // stop all trajectories of an instance at its first solution
    double eps;
    double tmax;
    const unsigned long long* deadline;  // %globaltimer deadline (device word); null = none
    void* slab;                  // global-storage mode: per-CTA trajectory storage
    long long slab_stride;       // values per CTA slab
};

// Cash-Karp tableau and NR step controller (AnalogSAT/cpu_sat/CpuRungeKutta.h:72-112).
namespace ck {
constexpr double TINY = 1e-20, SAFETY = 0.9, PGROW = -0.2, PSHRNK = -0.25, ERRCON = 1.89e-4,
                 HFACTOR = 0.1;
constexpr double b21 = 0.2, b31 = 3.0 / 40.0, b32 = 9.0 / 40.0, b41 = 0.3, b42 = -0.9, b43 = 1.2,
                 b51 = -11.0 / 54.0, b52 = 2.5, b53 = -70.0 / 27.0, b54 = 35.0 / 27.0,
                 b61 = 1631.0 / 55296.0, b62 = 175.0 / 512.0, b63 = 575.0 / 13824.0,
                 b64 = 44275.0 / 110592.0, b65 = 253.0 / 4096.0, c1 = 37.0 / 378.0,
                 c3 = 250.0 / 621.0, c4 = 125.0 / 594.0, c6 = 512.0 / 1771.0,
                 dc5 = -277.0 / 14336.0, dc1 = c1 - 2825.0 / 27648.0, dc3 = c3 - 18575.0 / 48384.0,
                 dc4 = c4 - 13525.0 / 55296.0, dc6 = c6 - 0.25;
}  // namespace ck

// FP32: y = x + h (sum_j b_j k_j), the sum formed left to right with fused
// multiply-adds in a fixed pattern (u = b_1 k_1; u = fma(b_j, k_j, u); y = fma(h, u, x)):
// explicit, so every kernel rounds the same way whatever the compiler would otherwise
// contract.  B holds the coefficients in order.
template <int NK>
__device__ __forceinline__ float fma_sum(const float (&b)[NK], const float (&k)[NK]) {
    float u = __fmul_rn(b[0], k[0]);
#pragma unroll
    for (int j = 1; j < NK; j++) u = __fmaf_rn(b[j], k[j], u);
    return u;
}
template <int NK>
__device__ __forceinline__ float fma_chain(const float (&b)[NK], const float (&k)[NK], float h, float x) {
    return __fmaf_rn(h, fma_sum<NK>(b, k), x);
}

// Stage input y_S = x + h * sum_j b_Sj k_j in the reference's expression order
// (FP64: every operation rounded as the reference rounds it; FP32: fma_chain).
template <int S, typename T>
__device__ __forceinline__ T stage_in(T x, T k1, T k2, T k3, T k4, T k5, T h) {
    using A = Arith<T>;
    if constexpr (S == 1) return x;
    if constexpr (sizeof(T) == 4) {
        if constexpr (S == 2) return __fmaf_rn(__fmul_rn((float)ck::b21, h), k1, x);
        if constexpr (S == 3) {
            const float b[2] = {(float)ck::b31, (float)ck::b32}, k[2] = {k1, k2};
            return fma_chain<2>(b, k, h, x);
        }
        if constexpr (S == 4) {
            const float b[3] = {(float)ck::b41, (float)ck::b42, (float)ck::b43}, k[3] = {k1, k2, k3};
            return fma_chain<3>(b, k, h, x);
        }
        if constexpr (S == 5) {
            const float b[4] = {(float)ck::b51, (float)ck::b52, (float)ck::b53, (float)ck::b54}, k[4] = {k1, k2, k3, k4};
            return fma_chain<4>(b, k, h, x);
        }
        if constexpr (S == 6) {
            const float b[5] = {(float)ck::b61, (float)ck::b62, (float)ck::b63, (float)ck::b64, (float)ck::b65},
                        k[5] = {k1, k2, k3, k4, k5};
            return fma_chain<5>(b, k, h, x);
        }
    }
    if constexpr (S == 2) return A::add(x, A::mul(A::mul(T(ck::b21), h), k1));
    if constexpr (S == 3) return A::add(x, A::mul(h, A::add(A::mul(T(ck::b31), k1), A::mul(T(ck::b32), k2))));
    if constexpr (S == 4)
        return A::add(x, A::mul(h, A::add(A::add(A::mul(T(ck::b41), k1), A::mul(T(ck::b42), k2)),
                                          A::mul(T(ck::b43), k3))));
    if constexpr (S == 5)
        return A::add(x, A::mul(h, A::add(A::add(A::add(A::mul(T(ck::b51), k1), A::mul(T(ck::b52), k2)),
                                                 A::mul(T(ck::b53), k3)),
                                          A::mul(T(ck::b54), k4))));
    if constexpr (S == 6)
        return A::add(
            x, A::mul(h, A::add(A::add(A::add(A::add(A::mul(T(ck::b61), k1), A::mul(T(ck::b62), k2)),
                                              A::mul(T(ck::b63), k3)),
                                       A::mul(T(ck::b64), k4)),
                                A::mul(T(ck::b65), k5))));
    return x;
}

// xnew = x + h (c1 k1 + c3 k3 + c4 k4 + c6 k6)
template <typename T>
__device__ __forceinline__ T rk_new(T x, T k1, T k3, T k4, T k6, T h) {
    using A = Arith<T>;
    if constexpr (sizeof(T) == 4) {
        const float b[4] = {(float)ck::c1, (float)ck::c3, (float)ck::c4, (float)ck::c6}, k[4] = {k1, k3, k4, k6};
        return fma_chain<4>(b, k, h, x);
    } else {
        return A::add(x, A::mul(h, A::add(A::add(A::add(A::mul(T(ck::c1), k1), A::mul(T(ck::c3), k3)),
                                                 A::mul(T(ck::c4), k4)),
                                          A::mul(T(ck::c6), k6))));
    }
}

// Error ratio |xerr / xscal| of one element (CpuRungeKutta.cpp:214, 233-235) with
// xscal = |x| + |k1 h0| + TINY (CpuRungeKutta.cpp:85).
// FP64 state: every operation rounded in the reference's order.
// FP32 state: formed in FP32 -- the k_j carry FP32 rounding already, so wider
// arithmetic here cannot sharpen the estimate; the max over elements and the
// controller run in FP64.  For log-space clause weights (u = log2 a) the scale is
// 1/ln2 + |k1 h0|: the reference's |a| + |h da/dt| expressed in u, i.e. the same
// relative error of a.
__device__ __forceinline__ double rk_err_ratio(double x, double k1, double k3, double k4, double k5,
                                               double k6, double h, double h0, bool) {
    using D = Arith<double>;
    const double e = D::mul(
        h, D::add(D::add(D::add(D::add(D::mul(ck::dc1, k1), D::mul(ck::dc3, k3)), D::mul(ck::dc4, k4)),
                         D::mul(ck::dc5, k5)),
                  D::mul(ck::dc6, k6)));
    const double sc = D::add(D::add(fabs(x), fabs(D::mul(k1, h0))), ck::TINY);
    return fabs(__ddiv_rn(e, sc));
}
__device__ __forceinline__ float rk_err_ratio(float x, float k1, float k3, float k4, float k5,
                                              float k6, float h, float h0, bool logw) {
    const float b[5] = {(float)ck::dc1, (float)ck::dc3, (float)ck::dc4, (float)ck::dc5, (float)ck::dc6},
                k[5] = {k1, k3, k4, k5, k6};
    const float e = __fmul_rn(h, fma_sum<5>(b, k));
    const float sc = __fadd_rn(__fadd_rn(logw ? kInvLn2 : fabsf(x), fabsf(__fmul_rn(k1, h0))), 1e-20f);
    return __fdividef(fabsf(e), sc);
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Persistent solver kernel
// ---------------------------------------------------------------------------
// Shared-memory layout of one trajectory (E = n + m state elements: internal
// variables 0..n-1, then clause weights n..n+m-1):
//   X, K1..K5   the RK stage vectors (state, k1..k5), E values each;
//   sy          the stage's spin vector plus the sentinel slot sy[n] = -1;
//   cs          SELL-32 contribution slots (nslots values, padding kept at 0).
// Element e is owned by thread e % blockDim.x in every stage loop, so stage vectors need no
// barriers; only sy and cs are exchanged between threads.
template <typename T>
struct Stages {
    T *X, *K1, *K2, *K3, *K4, *K5;
};

__host__ __device__ inline size_t solve_smem_values(int n, int m, int nslots) {
    const size_t E = (size_t)((n + m + 3) & ~3);
    return 6 * E + (size_t)((n + 1 + 3) & ~3) + (size_t)nslots + 1;
}

template <typename T, bool LOGA, int KMAX, bool EXACT, int ENC, int CL>
struct Solver {
    using A = Arith<T>;
    using ET = T;  // error-ratio type (see rk_err_ratio)

    // One RHS evaluation at stage S.  The stage input is formed on the fly from the
    // stage vectors; the derivative lands in K_S, or for S == 6 is consumed at once
    // into xnew (stored in K2, dead after the stage-6 input) and the error norm.
    // red_b: one slot per warp for the clause-weight sum of the bias term (CL == 1).
    template <int S>
    static __device__ __forceinline__ void eval(const Grp<CL>& g, const DevInstance& I, T* sy, T* cs, T knorm,
                                                const Stages<T>& st, T hT, T h0T, ET& errmax, double* red_b) {
        const int tid = g.gtid, nt = g.gnt;
        const int n = I.n;
        const bool bias = bias_on(I);
        double asum = 0.0;
        for (int v = tid; v < n; v += nt)
            sy[v] = stage_in<S>(st.X[v], st.K1[v], st.K2[v], st.K3[v], st.K4[v], st.K5[v], hT);
        g.sync();
        for (int m = tid; m < I.m; m += nt) {
            const int e = n + m;
            const T x = st.X[e];
            const T y = stage_in<S>(x, st.K1[e], st.K2[e], st.K3[e], st.K4[e], st.K5[e], hT);
            T am;
            if constexpr (LOGA) am = exp2_fast(y);
            else am = y;
            const T d = clause_phase<T, LOGA, KMAX, EXACT, ENC>(I, m, sy, cs, am, knorm);
            if (bias) asum += (double)am;
            if constexpr (S == 1) st.K1[e] = d;
            if constexpr (S == 2) st.K2[e] = d;
            if constexpr (S == 3) st.K3[e] = d;
            if constexpr (S == 4) st.K4[e] = d;
            if constexpr (S == 5) st.K5[e] = d;
            if constexpr (S == 6) {
                const T k1 = st.K1[e], k3 = st.K3[e], k4 = st.K4[e];
                errmax = fmax(errmax, rk_err_ratio(x, k1, k3, k4, st.K5[e], d, hT, h0T, LOGA));
                st.K2[e] = rk_new<T>(x, k1, k3, k4, d, hT);
            }
        }
        T bf = T(0);
        if (bias) {  // per-warp partial sums, read back by every thread after the barrier
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) asum += __shfl_xor_sync(0xffffffffu, asum, o);
            if ((threadIdx.x & 31) == 0) red_b[threadIdx.x >> 5] = asum;
        }
        g.sync();
        if (bias) {
            double tot = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += red_b[w];
            bf = bias_factor<T>(I, tot, knorm);
        }
        for (int v = tid; v < n; v += nt) {
            T d = var_phase<T>(I, v, cs);
            if (bias) d = Arith<T>::add(d, bias_term(bf, sy[v]));
            if constexpr (S == 1) st.K1[v] = d;
            if constexpr (S == 2) st.K2[v] = d;
            if constexpr (S == 3) st.K3[v] = d;
            if constexpr (S == 4) st.K4[v] = d;
            if constexpr (S == 5) st.K5[v] = d;
            if constexpr (S == 6) {
                const T x = st.X[v], k1 = st.K1[v], k3 = st.K3[v], k4 = st.K4[v];
                errmax = fmax(errmax, rk_err_ratio(x, k1, k3, k4, st.K5[v], d, hT, h0T, false));
                st.K2[v] = rk_new<T>(x, k1, k3, k4, d, hT);
            }
        }
    }
};

// Any block size that is a multiple of 32 and at most 1024 works; the host picks it
// so that every thread handles about the same number of clauses.
// GS = false: the trajectory lives in shared memory (compact literal words).
// GS = true:  "global storage" mode for instances too large for one SM's shared
//             memory: the same layout in a slab of global memory per trajectory in
//             flight (L2 resident when the active slabs fit), wide literal words.
// CL > 1 (global storage only): a thread-block cluster of CL CTAs on different SMs
//             works on one trajectory, synchronised by cluster barriers, so a few
//             very large trajectories still occupy the whole GPU.
template <typename T, bool LOGA, int KMAX, bool EXACT, bool GS, int CL>
__global__ void __launch_bounds__(1024, 1) solve_kernel(SolveParams P) {
    static_assert(CL == 1 || GS, "clusters share a trajectory through global memory");
    using A = Arith<T>;
    constexpr int ENC = GS ? 1 : 0;
    using S = Solver<T, LOGA, KMAX, EXACT, ENC, CL>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_d[36];
    __shared__ double red_b[32];
    __shared__ int red_i[33];
    __shared__ int s_unit, s_flag;
    const Grp<CL> g;
    const int tid = g.gtid, nt = g.gnt;
    const long long slot = blockIdx.x / CL;  // trajectory slot of this CTA (or cluster)

    while (true) {
        const int u = g.bcast(&s_unit, tid == 0 ? atomicAdd(P.queue_head, 1) : 0);
        if (u >= P.num_units) break;
        const int pidx = P.unit_inst[u];
        // an instance already solved by another trajectory (stop_on_first) is skipped,
        // its state left as it was set
        if (g.bcast(&s_flag, tid == 0 && P.stop_on_first ? (atomicAdd(P.inst_solved + pidx, 0) != 0 ? 1 : 0) : 0)) {
            if (tid == 0) {
                UnitResult r;
                r.time = 0.0; r.hdid = 0.0; r.status = SAT_ODE_INTERRUPTED; r.steps = 0; r.attempts = 0;
                r.rhs = 0; r.viol = -1; r.min_viol = -1;
                r.pad0 = r.pad1 = 0;
                P.results[u] = r;
            }
            g.sync();  // s_unit / s_flag are reused by the next unit
            continue;
        }
        const DevInstance I = P.inst[pidx];
        const int n = I.n, E = I.n + I.m;
        const int Ep = (E + 3) & ~3;
        T* base = GS ? reinterpret_cast<T*>(P.slab) + slot * P.slab_stride
                     : reinterpret_cast<T*>(smem_raw);
        Stages<T> st{base, base + Ep, base + 2 * Ep, base + 3 * Ep, base + 4 * Ep, base + 5 * Ep};
        T* sy = base + 6 * Ep;
        T* cs = sy + ((n + 1 + 3) & ~3);
        T* G = reinterpret_cast<T*>(P.states) + P.unit_state[u];
        const T knorm = (T)ldexp(1.0, -I.k);

        // initial state: public spins scattered to internal order; a -> log2 a
        for (int i = tid; i < n; i += nt) st.X[__ldg(I.iperm + i)] = G[i];
        for (int j = tid; j < I.m; j += nt) {
            const T a = G[n + j];
            const int e = n + __ldg(I.icperm + j);
            if constexpr (LOGA) st.X[e] = log2f(a);
            else st.X[e] = a;
        }
        for (int j = tid; j <= I.nslots; j += nt) cs[j] = T(0);
        if (tid == 0) sy[n] = T(-1);  // sentinel spin: padding literals are always FALSE
        g.sync();  // the scatter above wrote elements that other threads own in the stage loops

        double t = 0.0, hnext = 1e-9, hdid = 0.0;
        int steps = 0, attempts = 0, rhs = 0, viol = -1, minviol = INT_MAX;
        int status = SAT_UNKNOWN;

        while (status == SAT_UNKNOWN && t < P.tmax && steps < P.maxsteps) {
            bool underflow = false, interrupted = false;
            int taken = 0;
            for (int b = 0; b < P.batch; b++) {
                // ---- CpuRungeKutta::Step, count = 1 ----
                T dummy = T(0);
                S::template eval<1>(g, I, sy, cs, knorm, st, T(0), T(0), dummy, red_b);
                rhs++;
                const double h0 = hnext;
                const T h0T = (T)h0;
                double h = hnext, ermax = 0.0;
                while (true) {
                    const T hT = (T)h;
                    T em = T(0);
                    S::template eval<2>(g, I, sy, cs, knorm, st, hT, h0T, em, red_b);
                    S::template eval<3>(g, I, sy, cs, knorm, st, hT, h0T, em, red_b);
                    S::template eval<4>(g, I, sy, cs, knorm, st, hT, h0T, em, red_b);
                    S::template eval<5>(g, I, sy, cs, knorm, st, hT, h0T, em, red_b);
                    S::template eval<6>(g, I, sy, cs, knorm, st, hT, h0T, em, red_b);
                    rhs += 5;
                    attempts++;
                    // step-size control (CpuRungeKutta.cpp:229-259): one thread evaluates
                    // pow() and broadcasts the new step size with the error norm
                    ermax = group_max_then<CL>(g, (double)em, red_d, [&](double emax) {
                        const double e = __ddiv_rn(emax, P.eps);
                        double hn;
                        if (e <= 1.0)
                            hn = e > ck::ERRCON ? __dmul_rn(__dmul_rn(ck::SAFETY, h), pow(e, ck::PGROW))
                                                : __dmul_rn(5.0, h);
                        else
                            hn = fmax(__dmul_rn(__dmul_rn(ck::SAFETY, h), pow(e, ck::PSHRNK)),
                                      __dmul_rn(ck::HFACTOR, h));
                        red_d[34] = hn;
                        // early exit between batch checks: another trajectory solved this
                        // instance, or the wall-clock budget ran out (no extra barrier).  A
                        // cluster evaluates fn in every CTA, so it keeps to the batch-end check
                        // (decided once and broadcast) to stay uniform.
                        bool quit = false;
                        if constexpr (CL == 1)
                            quit = (P.stop_on_first && atomicAdd(P.inst_solved + pidx, 0) != 0) ||
                                   (P.deadline && globaltimer_ns() >= *P.deadline);
                        red_d[35] = quit ? 1.0 : 0.0;
                        return e;
                    });
                    const double hn = red_d[34];
                    if (red_d[35] != 0.0) { interrupted = true; break; }
                    if (ermax <= 1.0) { hnext = hn; break; }
                    h = hn;
                    if (__dadd_rn(t, h) == t) { underflow = true; break; }
                }
                if (underflow || interrupted) break;
                hdid = h;
                t = __dadd_rn(t, h);
                taken++;
                // accept: xnew (held in K2) becomes the state
                T* tmp = st.X; st.X = st.K2; st.K2 = tmp;
            }
            if (underflow) { status = SAT_UNDERFLOW; break; }
            steps += taken;
            if (interrupted) { status = SAT_ODE_INTERRUPTED; break; }

            // ---- CpuSat::GetClauseViolationCount on the accepted state ----
            for (int v = tid; v < n; v += nt) sy[v] = st.X[v];
            g.sync();
            int cnt = 0;
            for (int m = tid; m < I.m; m += nt) cnt += clause_violated<KMAX, EXACT, ENC>(I, m, sy);
            viol = group_sum<CL>(g, cnt, red_i);
            if (viol < minviol) {
                minviol = viol;
                if (P.best_bits) {
                    uint32_t* bits = P.best_bits + P.unit_bits[u];
                    for (int i0 = tid & ~31; i0 < n; i0 += nt) {
                        const int i = i0 + (tid & 31);
                        const bool bb = i < n && sy[__ldg(I.iperm + (i < n ? i : 0))] > T(0);
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
        for (int i = tid; i < n; i += nt) G[i] = st.X[__ldg(I.iperm + i)];
        for (int j = tid; j < I.m; j += nt) {
            const T v = st.X[n + __ldg(I.icperm + j)];
            if constexpr (LOGA) G[n + j] = exp2f(v);
            else G[n + j] = v;
        }
        if (tid == 0) {
            UnitResult r;
            r.time = t; r.hdid = hdid; r.status = status; r.steps = steps; r.attempts = attempts;
            r.rhs = rhs; r.viol = viol; r.min_viol = minviol == INT_MAX ? -1 : minviol;
            r.pad0 = r.pad1 = 0;
            P.results[u] = r;
        }
        g.sync();  // s_unit / shared buffers are reused by the next unit
    }
}

// ---------------------------------------------------------------------------
// Standalone batched RHS: one CTA per state, states in global memory (public
// layout).  Reads of x and writes of dxdt are coalesced; the permutation to the
// internal variable order happens in shared memory.
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t rhs_smem_values(int n, int m, int nslots) {
    return (size_t)((n + 1 + 3) & ~3) + (size_t)((m + 3) & ~3) + (size_t)nslots + 1;
}

template <typename T, bool LOGA, int KMAX, bool EXACT, int BT, bool GS>
__global__ void __launch_bounds__(BT) rhs_batch_kernel(DevInstance I, const T* __restrict__ x,
                                                        T* __restrict__ dxdt, int ntraj,
                                                        long long stride, T* slab,
                                                        long long slab_stride) {
    constexpr int ENC = GS ? 1 : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_b[BT / 32];
    T* sy = GS ? slab + (long long)blockIdx.x * slab_stride : reinterpret_cast<T*>(smem_raw);
    T* ab = sy + ((I.n + 1 + 3) & ~3);  // clause weights in internal clause order
    T* cs = ab + ((I.m + 3) & ~3);
    const int tid = threadIdx.x;
    const int n = I.n;
    const T knorm = (T)ldexp(1.0, -I.k);
    for (int j = tid; j <= I.nslots; j += BT) cs[j] = T(0);
    for (int tr = blockIdx.x; tr < ntraj; tr += gridDim.x) {
        const T* X = x + (long long)tr * stride;
        T* D = dxdt + (long long)tr * stride;
        // coalesced reads, permuted into the internal orders in shared memory
        for (int i = tid; i < n; i += BT) sy[__ldg(I.iperm + i)] = X[i];
        for (int j = tid; j < I.m; j += BT) ab[__ldg(I.icperm + j)] = X[n + j];
        if (tid == 0) sy[n] = T(-1);
        __syncthreads();
        const bool bias = bias_on(I);
        double asum = 0.0;
        for (int m = tid; m < I.m; m += BT) {
            const T a = ab[m];
            T am;
            if constexpr (LOGA) am = exp2_fast(a);
            else am = a;
            ab[m] = clause_phase<T, LOGA, KMAX, EXACT, ENC>(I, m, sy, cs, am, knorm);
            if (bias) asum += (double)am;
        }
        if (bias) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) asum += __shfl_xor_sync(0xffffffffu, asum, o);
            if ((tid & 31) == 0) red_b[tid >> 5] = asum;
        }
        __syncthreads();
        T bf = T(0);
        if (bias) {
            double tot = 0.0;
            for (int w = 0; w < BT / 32; w++) tot += red_b[w];
            bf = bias_factor<T>(I, tot, knorm);
        }
        // ds in internal order -> sy (no longer read) -> public order, coalesced; the
        // bias term reads the stage spin of its own element before overwriting it
        for (int v = tid; v < n; v += BT) {
            T d = var_phase<T>(I, v, cs);
            if (bias) d = Arith<T>::add(d, bias_term(bf, sy[v]));
            sy[v] = d;
        }
        __syncthreads();
        for (int i = tid; i < n; i += BT) D[i] = sy[__ldg(I.iperm + i)];
        for (int j = tid; j < I.m; j += BT) D[n + j] = ab[__ldg(I.icperm + j)];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Standalone batched RHS, two states per CTA pass (FP32): the spins and the clause
// contributions are held as float2 pairs, so the literal loads, index arithmetic and
// loop control are shared by the two states and the arithmetic runs as packed FP32x2
// (FFMA2/FMUL2/FADD2).  Products are formed in the one-state kernel's order (2 r =
// (km knorm)(2 a) is exact scaling).
//
// Data movement: two consecutive public states (contiguous in HBM) arrive in a shared
// staging buffer with one 1-D bulk copy (cp.async.bulk, mbarrier completion) that is
// issued one pair ahead by lane 0 of the last warp; the < 16-byte ragged ends of a row
// pair that does not start on a 16-byte boundary are fetched with plain loads.  The kernel then works in the
// public layout in place: a_m is read from and da_m written to its public position
// (the pair packing makes the 32 clauses of a warp hit 32 different banks there), ds
// is scattered to the public spin positions, and the finished pair leaves with one
// bulk store (when dxdt and x are congruent mod 16 bytes; plain coalesced stores
// otherwise).  Two staging buffers alternate: pair i is stored from one while pair
// i+1 lands in the other.  Two barriers per pair: one after the clause phase, one after
// the variable phase, which also permutes the next pair's spins (its buffer has landed).  A wait that does not complete within two seconds (it
// cannot, short of a broken device) turns every output of the CTA's remaining pairs
// into NaN and sets *status to 1 instead of hanging.
// Shared layout: 2 mbarriers | staging[2] (2 stride + 3 floats each) | sy2 | cs2.
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t rhs2_stage_floats(long long stride) {
    return (size_t)((2 * stride + 3 + 3) & ~3ll);
}
__host__ __device__ inline size_t rhs2_smem_bytes(int n, int m, int nslots) {
    return 16 + 8 * rhs2_stage_floats((long long)n + m) +
           8 * ((size_t)((n + 1 + 3) & ~3) + (size_t)nslots + 1);
}

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase `parity` of b to complete; false after `ns` nanoseconds.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* b, uint32_t parity, unsigned long long ns) {
    if (mbar_test(b, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_test(b, parity))
        if (globaltimer_ns() - t0 > ns) return false;
    return true;
}
// 1-D bulk copy global -> shared, completion counted on b (no multicast).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(b))
        : "memory");
}

// 1-D bulk copy shared -> global in the CTA's bulk group; the source must stay
// unchanged until bulk_wait_read() returns.
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"(smem_addr(src)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Row pair `pr` of x as it lands in the staging buffer: stg[off + e] = x[2 pr stride + e].
struct PairCopy {
    const float* src;
    int cnt;   // floats (one or two rows)
    int off;   // staging offset, keeps shared and global addresses congruent mod 16
    int head;  // plain-loaded floats before the first 16-byte boundary
    int nb;    // floats moved by the bulk copy (multiple of 4)
    __device__ PairCopy(const float* x, int pr, int ntraj, long long stride) {
        src = x + (long long)(2 * pr) * stride;
        cnt = (int)((2 * pr + 1 < ntraj ? 2 : 1) * stride);
        const uint32_t mis = (uint32_t)(reinterpret_cast<uintptr_t>(src) & 15u);
        off = (int)(mis >> 2);
        head = min(cnt, (int)(((16u - mis) & 15u) >> 2));
        nb = ((cnt - head) >> 2) << 2;
    }
    // thread t < 6 owns one ragged float: t < 3 in the head, 3..5 in the tail
    __device__ int ragged(int t) const {
        const int e = t < 3 ? t : head + nb + (t - 3);
        return (t < 3 ? e < head : e < cnt) ? e : -1;
    }
};

// CPT / VPT: clauses / variables per thread (M <= CPT * BT, N <= VPT * BT); a thread's
// literal words, public clause and variable indices and SELL rows are the same for
// every pair, so they are loaded once into registers.
template <bool LOGA, int KMAX, bool EXACT, int BT, int CPT, int VPT>
__global__ void __launch_bounds__(BT, 1) rhs_pair_kernel(DevInstance I, const float* __restrict__ x,
                                                          float* __restrict__ dxdt, int ntraj,
                                                          long long stride, int bulk_out,
                                                          int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
    const size_t sf = rhs2_stage_floats(stride);
    float* stg0 = reinterpret_cast<float*>(smem_raw + 16);
    float2* sy = reinterpret_cast<float2*>(stg0 + 2 * sf);
    float2* cs = sy + ((I.n + 1 + 3) & ~3);
    const int tid = threadIdx.x;
    const int n = I.n;
    const float knorm = (float)ldexp(1.0, -I.k);
    const float2 kn2 = f2(knorm);
    const int npairs = (ntraj + 1) / 2;
    const int G = gridDim.x;
    constexpr unsigned long long kWaitNs = 2000000000ull;
    int pr = blockIdx.x;
    if (pr >= npairs) return;
    for (int j = tid; j <= I.nslots; j += BT) cs[j] = f2(0.0f);
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    Lit<0> lw[CPT][KMAX];
    int lj[CPT];
#pragma unroll
    for (int i = 0; i < CPT; i++) {
        const int m = tid + i * BT;
        lj[i] = m < I.m ? n + ld_ro(I.cperm + m) : 0;
#pragma unroll
        for (int q = 0; q < KMAX; q++)
            if (m < I.m && (EXACT || q < I.k)) lw[i][q].load(I, q * I.mp + m);
            else lw[i][q].w = 0;
    }
    int vp[VPT];
    uint32_t vrows[VPT];  // first row | end row << 16 (rows < 2048 for compact instances)
#pragma unroll
    for (int i = 0; i < VPT; i++) {
        const int v = tid + i * BT;
        vp[i] = v < n ? __ldg(I.perm + v) : 0;
        vrows[i] = v < n ? (uint32_t)ld_ro(I.srow + (v >> 5)) | ((uint32_t)ld_ro(I.srow + (v >> 5) + 1) << 16) : 0u;
    }
    if (tid == 0) sy[n] = f2(-1.0f);
    __syncthreads();
    // All bulk copies and stores are issued by lane 0 of the last warp (IO), so that the
    // store -> reuse wait falls on a warp with no more clauses than the first.  Copy of
    // pair q into buffer b: IO starts the bulk part; after it, lanes 0..5 of the same
    // warp load the < 16-byte ragged ends and store them into the buffer (positions the
    // bulk copy does not write).  The buffer's previous pair has left it by then: IO
    // waited for its bulk store to read out, and __syncwarp orders the lanes after it.
    constexpr int IO = BT - 32;
    const bool io_warp = tid >= IO;
    auto issue = [&](int q, int b) {
        const PairCopy c(x, q, ntraj, stride);
        float* dst = stg0 + (size_t)b * sf;
        if (tid == IO) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive_tx(bar + b, (uint32_t)c.nb * 4u);
            if (c.nb > 0) bulk_load(dst + c.off + c.head, c.src + c.head, (uint32_t)c.nb * 4u, bar + b);
        }
        if ((unsigned)(tid - IO) < 6u) {  // lanes 0..5 of the IO warp
            const int e = c.ragged(tid - IO);
            if (e >= 0) dst[c.off + e] = __ldg(c.src + e);
        }
    };
    // Spins of the pair in buffer b into internal order, interleaved.
    auto permute = [&](int q, int b) {
        const PairCopy c(x, q, ntraj, stride);
        const float* A0 = stg0 + (size_t)b * sf + c.off;
        const float* A1 = 2 * q + 1 < ntraj ? A0 + stride : A0;
#pragma unroll
        for (int i = 0; i < VPT; i++)
            if (tid + i * BT < n) sy[tid + i * BT] = make_float2(A0[vp[i]], A1[vp[i]]);
    };
    uint32_t parity = 0;   // bit b: phase parity expected next on bar[b]
    uint32_t pending = 1;  // bit b: a copy into buffer b not yet waited for (same in all threads)
    if (io_warp) issue(pr, 0);
    if (pr + G < npairs) {
        if (io_warp) issue(pr + G, 1);
        pending |= 2u;
    }
    bool ok = mbar_wait_for(bar, 0, kWaitNs);
    parity ^= 1u;
    pending &= ~1u;
    __syncthreads();  // the ragged ends stored by the IO warp
    permute(pr, 0);
    bool failed = __syncthreads_or(!ok);
    // Per pair: clause phase | barrier | next pair's copy waited for | variable phase of
    // this pair and spin permutation of the next (independent work in one phase) |
    // barrier + timeout vote | this pair stored, the pair after next copied in.
    for (int it = 0; !failed && pr < npairs; pr += G, it++) {
        const int b = it & 1;
        const bool two = 2 * pr + 1 < ntraj;
        const PairCopy cur(x, pr, ntraj, stride);
        float* S0 = stg0 + (size_t)b * sf + cur.off;
        float* S1 = two ? S0 + stride : S0;
        // clause phase: a_m in, da_m out at the public clause position
#pragma unroll
        for (int i = 0; i < CPT; i++) {
            if (tid + i * BT >= I.m) break;
            const Lit<0>* w = lw[i];
            float2 f[KMAX];
            float2 km = kn2;
            const int j = lj[i];
#pragma unroll
            for (int q = 0; q < KMAX; q++) {
                if (EXACT || q < I.k) {
                    // c = -c_lit = +1 for a negated literal, -1 otherwise (from the sign bit):
                    // f = 1 - c_lit s = 1 + c s
                    const float c = __int_as_float((w[q].w & 0x80000000u) ^ 0xBF800000u);
                    f[q] = __ffma2_rn(f2(c), sy[w[q].var()], f2(1.0f));
                    km = __fmul2_rn(km, f[q]);
                }
            }
            const float2 a = make_float2(S0[j], S1[j]);
            float2 am;
            if constexpr (LOGA) am = make_float2(exp2_fast(a.x), exp2_fast(a.y));
            else am = a;
            // da: (km km) / ln 2 in log space, (a km) km otherwise, as in the one-state kernel
            const float2 da = LOGA ? __fmul2_rn(__fmul2_rn(km, km), f2(kInvLn2))
                                   : __fmul2_rn(__fmul2_rn(am, km), km);
            S0[j] = da.x;
            S1[j] = da.y;
            // -2 r (exact scaling): the contribution c_lit 2 r K_mi is then (-2 r K_mi) c
            const float2 r2n = __fmul2_rn(__fmul2_rn(km, kn2), __fmul2_rn(am, f2(-2.0f)));
#pragma unroll
            for (int q = 0; q < KMAX; q++) {
                if (EXACT || q < I.k) {
                    float2 prod = f2(1.0f);
                    bool first = true;
#pragma unroll
                    for (int l = 0; l < KMAX; l++) {
                        if (l != q && (EXACT || l < I.k)) {
                            prod = first ? f[l] : __fmul2_rn(prod, f[l]);
                            first = false;
                        }
                    }
                    const float c = __int_as_float((w[q].w & 0x80000000u) ^ 0xBF800000u);
                    cs[w[q].slot()] = __fmul2_rn(__fmul2_rn(r2n, prod), f2(c));
                }
            }
        }
        __syncthreads();
        const bool more = pr + G < npairs;
        ok = true;
        if (more) {
            ok = mbar_wait_for(bar + (b ^ 1), (parity >> (b ^ 1)) & 1u, kWaitNs);
            parity ^= 1u << (b ^ 1);
            pending &= ~(1u << (b ^ 1));
        }
        // var phase: ds_i to the public spin position
#pragma unroll
        for (int i = 0; i < VPT; i++) {
            const int v = tid + i * BT;
            if (v >= n) break;
            const int r0 = (int)(vrows[i] & 0xffffu), r1 = (int)(vrows[i] >> 16);
            const float2* p = cs + r0 * 32 + (v & 31);
            float2 sum = f2(0.0f);
#pragma unroll 8
            for (int r = r0; r < r1; r++, p += 32) sum = __fadd2_rn(sum, *p);
            S0[vp[i]] = sum.x;
            S1[vp[i]] = sum.y;
        }
        // the next pair's spins (its buffer is the other one; sy is free: this pair's
        // clause phase has read it)
        if (more) permute(pr + G, b ^ 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // results -> bulk store
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        float* D = dxdt + (long long)(2 * pr) * stride;
        if (bulk_out) {
            if (tid == IO && cur.nb > 0) bulk_store(D + cur.head, S0 + cur.head, (uint32_t)cur.nb * 4u);
            if ((unsigned)(tid - IO) < 6u) {
                const int e = cur.ragged(tid - IO);
                if (e >= 0) D[e] = S0[e];
            }
        } else {
            for (int e = tid; e < cur.cnt; e += BT) D[e] = S0[e];
            __syncthreads();  // the buffer is read out before the copy into it
        }
        if (pr + 2 * G < npairs) {
            // this buffer takes the pair after next once its store has read it out
            if (io_warp) {
                if (tid == IO && bulk_out) bulk_wait_read();
                __syncwarp();
                issue(pr + 2 * G, b);
            }
            pending |= 1u << b;
        }
        // no barrier here: the next writes to this buffer (the copy above, after the
        // store's read), to sy (next variable phase) and to cs (next clause phase) all
        // come after the next barriers
    }
    if (!failed) {
        if (tid == IO) bulk_wait_all();
        return;
    }
    // a copy did not land within the limit (it cannot, short of a broken device): let
    // the copies still in flight land, wait for this CTA's stores, flag the error and
    // turn every output of the CTA's remaining pairs into NaN
    for (int b = 0; b < 2; b++)
        if (pending & (1u << b)) mbar_wait_for(bar + b, (parity >> b) & 1u, kWaitNs);
    if (tid == IO) {
        bulk_wait_all();
        atomicExch(status, 1);
    }
    const float nan = __int_as_float(0x7fc00000);
    for (; pr < npairs; pr += G) {
        const long long cnt = (2 * pr + 1 < ntraj ? 2 : 1) * stride;
        for (long long e = tid; e < cnt; e += BT) dxdt[(long long)(2 * pr) * stride + e] = nan;
    }
}

// Exact unsat counts of many states: one CTA per state.
template <typename T, int KMAX, bool EXACT, int BT, bool GS>
__global__ void __launch_bounds__(BT) viol_batch_kernel(DevInstance I, const T* __restrict__ x,
                                                         int* __restrict__ counts, int ntraj,
                                                         long long stride, T* slab,
                                                         long long slab_stride) {
    constexpr int ENC = GS ? 1 : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int red_i[32];
    T* sy = GS ? slab + (long long)blockIdx.x * slab_stride : reinterpret_cast<T*>(smem_raw);
    const int tid = threadIdx.x;
    for (int tr = blockIdx.x; tr < ntraj; tr += gridDim.x) {
        const T* X = x + (long long)tr * stride;
        for (int i = tid; i < I.n; i += BT) sy[__ldg(I.iperm + i)] = X[i];
        if (tid == 0) sy[I.n] = T(-1);
        __syncthreads();
        int cnt = 0;
        for (int m = tid; m < I.m; m += BT) cnt += clause_violated<KMAX, EXACT, ENC>(I, m, sy);
        cnt = block_sum(cnt, red_i);
        if (tid == 0) counts[tr] = cnt;
        __syncthreads();
    }
}

}  // namespace asb
