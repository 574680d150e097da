// Streamed RK45 solver for instances too large for one SM ("stream" storage mode).
//
// The same integrator as solve_kernel (SatSolver::DoSolve + CpuRungeKutta::Step/rkqs/
// rkck + CpuSat::GetDerivatives / GetClauseViolationCount: AnalogSAT/solver/
// SatSolver.h:273-355, AnalogSAT/cpu_sat/CpuRungeKutta.cpp:66-100,181-267,
// AnalogSAT/cpu_sat/CpuSat.cpp:65-94,136-173,199-241), reorganised for the whole GPU:
//
//  * Trajectories of one instance are grouped by eight ("lanes").  Every per-element
//    vector of a group is stored interleaved, [element][lane], so an FP32 element row
//    is one whole 32-byte sector: a random spin gather or a contribution access moves
//    no byte it does not use, and one pass over the literal words serves eight
//    trajectories.  Two adjacent threads share a row, four lanes each, which keeps
//    a thread's registers at four lanes' worth.
//  * A group's vectors live in HBM: state X, stage derivatives K1..K5 (K2 doubles as
//    the candidate state xnew after stage 6), stage spins SY (+ the sentinel row n,
//    pinned at -1) and the literal contributions CS, clause-major ([slot q][clause]),
//    so the clause kernel writes whole lines: scattered 16-byte partial-sector writes
//    (the SELL slot order of the shared-memory kernels) cost as much as the whole rest
//    of a pass here.  The variable kernel gathers a variable's contributions through
//    its occurrence list (CSR, public clause order: the reference's summation order).
//  * One "pass" is one RK attempt of every lane: per stage S = 1..6 a clause kernel
//    (stage input of the clause weights, spin gathers, K_m, contributions into CS,
//    da -> K_S) and a variable kernel (occurrence-list sums -> K_S, spin input of
//    stage S+1).  Optionally (as_solver_set_stream_parts) the clauses are split into
//    parts by public index, each part's clause kernel followed at once by a variable
//    kernel that continues the row sums over that part's occurrences (the sums still
//    run in public clause order), so CS is read back from L2.
//    The kernels are launched group by group, so a group's CS is written and read
//    back while much of it is still in L2.
//  * Each lane keeps its own step size, time, counters and status.  A lane whose
//    previous attempt was rejected recomputes k1 at the same state (identical values)
//    and retries with its smaller step; counters follow the reference (1 + 5 per
//    attempt RHS evaluations per step, steps counted per completed batch).
//  * The accept/reject decision is taken by the last block of the stage-6 variable
//    kernel (ticket counter, no waiting); the post kernel commits accepted states,
//    counts unsat clauses for lanes at a batch end and applies SatSolver's status
//    rules in its last block.  No kernel waits on another block.
// Per-lane arithmetic mirrors clause_phase / var_phase / stage_in / rk_new /
// rk_err_ratio and the controller of solve_kernel operation for operation; with the
// explicitly rounded FP64 arithmetic a lane follows solve_kernel's trajectory bit for
// bit on the same packing (tested).
#pragma once

#include "as_kernels.cuh"

namespace asb {

#ifndef AS_STREAM_LANES
#define AS_STREAM_LANES 8
#endif
constexpr int kLanes = AS_STREAM_LANES;  // trajectories per stream group
constexpr int kSub = 4;                  // lanes per thread in the clause and variable kernels
constexpr int kRowThreads = kLanes / kSub;  // threads sharing an element row
static_assert(kLanes % kSub == 0 && kRowThreads <= 32 && (kRowThreads & (kRowThreads - 1)) == 0, "lane split");

struct LaneState {
    double t, h, h0, hnext, hdid;
    unsigned long long err;  // max error ratio of the attempt (non-negative double bits)
    int steps, taken, attempts, rhs, viol, minviol, status;
    int acc;       // last attempt accepted: K2 holds the new state until the post kernel
    int check;     // batch end reached: unsat count due in the post kernel
    int newstep;   // next attempt starts a new step (h = h0 = hnext, one more RHS)
    int vcount;    // unsat count accumulator
    int unit;      // solver unit (launch order) of this lane, -1 for a padding lane
};

// Device view of one group.  Pointers address [rows][kLanes] arrays of T.
template <typename T>
struct StreamArgs {
    DevInstance I;
    T *X, *K1, *K2, *K3, *K4, *K5, *SY, *CS;
    T* ACC;                 // [n][kLanes] partial row sums between clause parts
    const int* vstart;      // this part's occurrence ranges: [vstart[v], vstart[n + v])
    const int* vpos;        // occurrences: CS row q * mp + m, public clause order
    int m0, m1;             // clause range of this part
    int part, nparts;
    LaneState* lanes;       // [kLanes]
    int* tickets;           // [2] last-block tickets (decision, post)
    int* active;            // lanes of the group still running
    uint32_t* cand_bits;    // [kLanes][words] assignment at the current batch check
    uint32_t* best_bits;    // solver best-assignment array (or null)
    const long long* unit_bits;  // [units] word offsets into best_bits
    int* inst_solved;       // stop-on-first flags [problems]
    const unsigned long long* deadline;  // %globaltimer deadline (or null)
    int pidx, S, batch, maxsteps, stop_on_first;
    double eps, tmax;
};

template <typename T> struct L4 { T v[kSub]; };

__device__ __forceinline__ L4<float> ld4(const float* p) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    return {{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ void st4(float* p, const L4<float>& a) {
    *reinterpret_cast<float4*>(p) = make_float4(a.v[0], a.v[1], a.v[2], a.v[3]);
}
__device__ __forceinline__ L4<double> ld4(const double* p) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(double* p, const L4<double>& a) {
    reinterpret_cast<double2*>(p)[0] = make_double2(a.v[0], a.v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(a.v[2], a.v[3]);
}

// Per-lane block max of non-negative values, a thread holding kSub lanes starting at
// lane (threadIdx.x % kRowThreads) * kSub, folded into lanes[l].err (atomicMax on the bit
// pattern, which orders non-negative doubles like their values).
__device__ __forceinline__ void lanes_max(const double (&v)[kSub], double* red, LaneState* lanes) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    double w[kSub];
#pragma unroll
    for (int l = 0; l < kSub; l++) {
        w[l] = v[l];
#pragma unroll
        for (int o = kRowThreads; o < 32; o <<= 1) w[l] = fmax(w[l], __shfl_xor_sync(0xffffffffu, w[l], o));
    }
    if (lane < kRowThreads)
#pragma unroll
        for (int l = 0; l < kSub; l++) red[(lane * kSub + l) * 32 + warp] = w[l];
    __syncthreads();
    if (threadIdx.x < kLanes) {
        double m = 0.0;
        for (int i = 0; i < nw; i++) m = fmax(m, red[threadIdx.x * 32 + i]);
        atomicMax(&lanes[threadIdx.x].err, (unsigned long long)__double_as_longlong(m));
    }
}

// Ticket of the block that finishes last (after its own global writes are fenced).
__device__ __forceinline__ bool last_block(int* ticket, int* s_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *s_flag = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
    __syncthreads();
    const bool last = *s_flag != 0;
    if (last) __threadfence();
    return last;
}

template <typename T>
__device__ __forceinline__ void load_lane_steps(const LaneState* L, T (&h)[kSub], T (&h0)[kSub]) {
#pragma unroll
    for (int l = 0; l < kSub; l++) {
        h[l] = (T)L[l].h;
        h0[l] = (T)L[l].h0;
    }
}

// Stage input of stage S for one element, per lane (S is uniform per launch).
template <typename T>
__device__ __forceinline__ T stage_lane(int S, T x, T k1, T k2, T k3, T k4, T k5, T h) {
    switch (S) {
        case 1: return x;
        case 2: return stage_in<2, T>(x, k1, k2, k3, k4, k5, h);
        case 3: return stage_in<3, T>(x, k1, k2, k3, k4, k5, h);
        case 4: return stage_in<4, T>(x, k1, k2, k3, k4, k5, h);
        case 5: return stage_in<5, T>(x, k1, k2, k3, k4, k5, h);
        default: return stage_in<6, T>(x, k1, k2, k3, k4, k5, h);
    }
}

// The stage vectors of one element that stage S reads (X, K1..K_{S-1}).
template <typename T>
struct StageRow {
    L4<T> x, k1, k2, k3, k4, k5;
    // i: index of the thread's first lane of the row ([row][lane] layout)
    __device__ __forceinline__ void load(const StreamArgs<T>& A, long long i, int S) {
        x = ld4(A.X + i);
        k1 = k2 = k3 = k4 = k5 = L4<T>{};
        if (S >= 2) k1 = ld4(A.K1 + i);
        if (S >= 3) k2 = ld4(A.K2 + i);
        if (S >= 4) k3 = ld4(A.K3 + i);
        if (S >= 5) k4 = ld4(A.K4 + i);
        if (S >= 6) k5 = ld4(A.K5 + i);
    }
    __device__ __forceinline__ L4<T> input(int S, const T (&h)[kSub]) const {
        L4<T> y;
#pragma unroll
        for (int l = 0; l < kSub; l++)
            y.v[l] = stage_lane<T>(S, x.v[l], k1.v[l], k2.v[l], k3.v[l], k4.v[l], k5.v[l], h[l]);
        return y;
    }
};

template <typename T>
__device__ __forceinline__ T* stage_out(const StreamArgs<T>& A, int S) {
    return S == 1 ? A.K1 : S == 2 ? A.K2 : S == 3 ? A.K3 : S == 4 ? A.K4 : A.K5;
}

// Stage S, clause side: a_m stage input, spin gathers, K_m and the leave-one-out
// products (clause_phase's expression order, per lane), contributions into CS,
// da_m -> K_S (stage 6: xnew -> K2 and the error ratio).  kRowThreads threads per
// clause, kSub lanes each.
template <typename T, bool LOGA, int KMAX, bool EXACT>
__global__ void __launch_bounds__(256) stream_clause_kernel(StreamArgs<T> A) {
    using Ar = Arith<T>;
    __shared__ double red[kLanes * 32];
    if (*A.active == 0) return;
    const DevInstance& I = A.I;
    const int S = A.S, n = I.n;
    const int lb = (threadIdx.x % kRowThreads) * kSub;  // first lane of this thread
    T h[kSub], h0[kSub];
    load_lane_steps(A.lanes + lb, h, h0);
    const T knorm = (T)ldexp(1.0, -I.k);
    double em[kSub] = {0.0, 0.0, 0.0, 0.0};
    T* KS = stage_out(A, S);
    const long long total = (long long)kRowThreads * (A.m1 - A.m0);
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < total;
         it += (long long)gridDim.x * blockDim.x) {
        const int m = A.m0 + (int)(it / kRowThreads);
        const long long i = ((long long)n + m) * kLanes + lb;
        StageRow<T> row;
        row.load(A, i, S);
        const L4<T> y = row.input(S, h);
        L4<T> am;
#pragma unroll
        for (int l = 0; l < kSub; l++) {
            if constexpr (LOGA) am.v[l] = exp2_fast(y.v[l]);
            else am.v[l] = y.v[l];
        }
        Lit<1> w[KMAX];
        T f[KMAX][kSub];
        T km[kSub];
#pragma unroll
        for (int l = 0; l < kSub; l++) km[l] = knorm;
#pragma unroll
        for (int q = 0; q < KMAX; q++) {
            if (EXACT || q < I.k) {
                w[q].load(I, q * I.mp + m);
                const L4<T> sv = ld4(A.SY + (long long)w[q].var() * kLanes + lb);
#pragma unroll
                for (int l = 0; l < kSub; l++) {
                    f[q][l] = w[q].neg() ? Ar::add(T(1), sv.v[l]) : Ar::sub(T(1), sv.v[l]);
                    km[l] = Ar::mul(km[l], f[q][l]);
                }
            }
        }
        L4<T> d;
#pragma unroll
        for (int l = 0; l < kSub; l++) {
            if constexpr (LOGA) d.v[l] = km[l] * km[l] * T(kInvLn2);
            else d.v[l] = Ar::mul(Ar::mul(am.v[l], km[l]), km[l]);
        }
        if (KMAX <= 10 || I.k <= 10) {
            T r[kSub];
#pragma unroll
            for (int l = 0; l < kSub; l++) r[l] = Ar::mul(Ar::mul(km[l], knorm), am.v[l]);
#pragma unroll
            for (int q = 0; q < KMAX; q++) {
                if (EXACT || q < I.k) {
                    L4<T> c;
#pragma unroll
                    for (int l = 0; l < kSub; l++) {
                        T prod = T(1);
                        bool first = true;
#pragma unroll
                        for (int j = 0; j < KMAX; j++) {
                            if (j != q && (EXACT || j < I.k)) {
                                prod = first ? f[j][l] : Ar::mul(prod, f[j][l]);
                                first = false;
                            }
                        }
                        T rr = Ar::mul(r[l], prod);
                        rr = rr + rr;
                        c.v[l] = w[q].neg() ? -rr : rr;
                    }
                    st4(A.CS + ((long long)q * I.mp + m) * kLanes + lb, c);
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < KMAX; q++) {
                if (EXACT || q < I.k) {
                    L4<T> c;
#pragma unroll
                    for (int l = 0; l < kSub; l++) {
                        T temp = km[l];
#pragma unroll
                        for (int j = 0; j < KMAX; j++)
                            if (EXACT || j < I.k) temp = Ar::mul(temp, j == q ? T(1) : f[j][l]);
                        const T rr = Ar::mul(Ar::mul(Ar::mul(T(2), temp), knorm), am.v[l]);
                        c.v[l] = w[q].neg() ? -rr : rr;
                    }
                    st4(A.CS + ((long long)q * I.mp + m) * kLanes + lb, c);
                }
            }
        }
        if (S < 6) {
            st4(KS + i, d);
        } else {
            L4<T> xn;
#pragma unroll
            for (int l = 0; l < kSub; l++) {
                em[l] = fmax(em[l], (double)rk_err_ratio(row.x.v[l], row.k1.v[l], row.k3.v[l], row.k4.v[l],
                                                         row.k5.v[l], d.v[l], h[l], h0[l], LOGA));
                xn.v[l] = rk_new<T>(row.x.v[l], row.k1.v[l], row.k3.v[l], row.k4.v[l], d.v[l], h[l]);
            }
            st4(A.K2 + i, xn);
        }
    }
    if (S == 6) lanes_max(em, red, A.lanes);
}

// The step-size controller of one lane after its attempt (solve_kernel's, itself
// CpuRungeKutta.cpp:218-267 + SatSolver.h:273-355 batch counting).
template <typename T>
__device__ __forceinline__ void lane_decide(LaneState& L, const StreamArgs<T>& A) {
    const double emax = __longlong_as_double((long long)L.err);
    L.err = 0ull;
    L.acc = 0;
    if (L.status != SAT_UNKNOWN) return;
    L.rhs += 5;
    L.attempts++;
    const double e = __ddiv_rn(emax, A.eps);
    const double h = L.h;
    double hn;
    if (e <= 1.0)
        hn = e > ck::ERRCON ? __dmul_rn(__dmul_rn(ck::SAFETY, h), pow(e, ck::PGROW)) : __dmul_rn(5.0, h);
    else
        hn = fmax(__dmul_rn(__dmul_rn(ck::SAFETY, h), pow(e, ck::PSHRNK)), __dmul_rn(ck::HFACTOR, h));
    // early exit between batch checks, as in solve_kernel: another trajectory solved
    // this instance, or the wall-clock budget ran out
    const bool quit = (A.stop_on_first && atomicAdd(A.inst_solved + A.pidx, 0) != 0) ||
                      (A.deadline && globaltimer_ns() >= *A.deadline);
    if (quit) {
        L.steps += L.taken;
        L.taken = 0;
        L.status = SAT_ODE_INTERRUPTED;
        return;
    }
    if (e <= 1.0) {
        L.hnext = hn;
        L.hdid = h;
        L.t = __dadd_rn(L.t, h);
        L.taken++;
        L.acc = 1;
        L.newstep = 1;
        if (L.taken == A.batch) {
            L.steps += L.taken;
            L.taken = 0;
            L.check = 1;
        }
    } else {
        L.h = hn;
        if (__dadd_rn(L.t, hn) == L.t) L.status = SAT_UNDERFLOW;
    }
}

// Stage S, variable side: occurrence-list sums -> K_S and the spin input of stage
// S + 1 (stage 6: xnew -> K2, the error ratio, and in the last block the lanes'
// decisions).  kRowThreads threads per variable, kSub lanes each.
template <typename T, bool LOGA>
__global__ void __launch_bounds__(256) stream_var_kernel(StreamArgs<T> A) {
    using Ar = Arith<T>;
    __shared__ double red[kLanes * 32];
    __shared__ int s_flag;
    if (*A.active == 0) return;
    const DevInstance& I = A.I;
    const int S = A.S, n = I.n;
    const int lb = (threadIdx.x % kRowThreads) * kSub;
    T h[kSub], h0[kSub];
    load_lane_steps(A.lanes + lb, h, h0);
    double em[kSub] = {0.0, 0.0, 0.0, 0.0};
    T* KS = stage_out(A, S);
    const long long total = (long long)kRowThreads * n;
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < total;
         it += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(it / kRowThreads);
        const long long i = (long long)v * kLanes + lb;
        const int r0 = __ldg(A.vstart + v), r1 = __ldg(A.vstart + n + v);
        L4<T> d;
        if (A.part > 0) {
            d = ld4(A.ACC + i);  // the sum so far, continued in the same order
        } else {
#pragma unroll
            for (int l = 0; l < kSub; l++) d.v[l] = T(0);
        }
#pragma unroll 8
        for (int r = r0; r < r1; r++) {
            const L4<T> c = ld4(A.CS + (long long)__ldg(A.vpos + r) * kLanes + lb);
#pragma unroll
            for (int l = 0; l < kSub; l++) d.v[l] = Ar::add(d.v[l], c.v[l]);
        }
        if (A.part + 1 < A.nparts) {
            st4(A.ACC + i, d);
            continue;
        }
        StageRow<T> row;
        if (S < 6) {
            st4(KS + i, d);
            // spin input of the next stage: K_S of this element was just formed
            row.load(A, i, S);
            if (S == 1) row.k1 = d;
            if (S == 2) row.k2 = d;
            if (S == 3) row.k3 = d;
            if (S == 4) row.k4 = d;
            if (S == 5) row.k5 = d;
            st4(A.SY + i, row.input(S + 1, h));
        } else {
            row.load(A, i, 6);
            L4<T> xn;
#pragma unroll
            for (int l = 0; l < kSub; l++) {
                em[l] = fmax(em[l], (double)rk_err_ratio(row.x.v[l], row.k1.v[l], row.k3.v[l], row.k4.v[l],
                                                         row.k5.v[l], d.v[l], h[l], h0[l], false));
                xn.v[l] = rk_new<T>(row.x.v[l], row.k1.v[l], row.k3.v[l], row.k4.v[l], d.v[l], h[l]);
            }
            st4(A.K2 + i, xn);
        }
    }
    if (S != 6 || A.part + 1 < A.nparts) return;
    lanes_max(em, red, A.lanes);
    if (!last_block(A.tickets, &s_flag)) return;
    if (threadIdx.x < kLanes) lane_decide(A.lanes[threadIdx.x], A);
    if (threadIdx.x == 0) A.tickets[0] = 0;
}

// After the decision: commit accepted states (X <- K2), spins of the next pass's
// stage 1 (SY <- X), unsat counts and the assignment of lanes at a batch end; the
// last block applies SatSolver's batch-end rules.  Block roles: [0, nbv) variables,
// [nbv, nbv + nbc) clauses, the rest 32-variable words of the public assignment.
template <typename T, int KMAX, bool EXACT>
__global__ void __launch_bounds__(256) stream_post_kernel(StreamArgs<T> A, int nbv, int nbc) {
    __shared__ int red[32 * kLanes];
    __shared__ int s_flag;
    __shared__ int s_improved[kLanes];
    if (*A.active == 0) return;
    const DevInstance& I = A.I;
    const int n = I.n, words = (n + 31) / 32;
    unsigned acc = 0, chk = 0;  // lane bit masks
#pragma unroll
    for (int l = 0; l < kLanes; l++) {
        acc |= (A.lanes[l].acc ? 1u : 0u) << l;
        chk |= (A.lanes[l].check ? 1u : 0u) << l;
    }
    // commit of one element row (vector accesses, kSub lanes each): lanes whose
    // attempt was accepted take K2; the committed row is returned in x
    auto commit = [&](long long row, L4<T> (&x)[kRowThreads]) {
#pragma unroll
        for (int c = 0; c < kRowThreads; c++) {
            const long long i = row * kLanes + c * kSub;
            x[c] = ld4(A.X + i);
            if ((acc >> (c * kSub)) & ((1u << kSub) - 1u)) {
                const L4<T> xn = ld4(A.K2 + i);
#pragma unroll
                for (int l = 0; l < kSub; l++)
                    if ((acc >> (c * kSub + l)) & 1u) x[c].v[l] = xn.v[l];
                st4(A.X + i, x[c]);
            }
        }
    };
    const int b = blockIdx.x;
    if (b < nbv) {
        for (int v = b * blockDim.x + threadIdx.x; v < n; v += nbv * blockDim.x) {
            L4<T> x[kRowThreads];
            commit(v, x);
#pragma unroll
            for (int c = 0; c < kRowThreads; c++) st4(A.SY + (long long)v * kLanes + c * kSub, x[c]);
        }
    } else if (b < nbv + nbc) {
        int cnt[kLanes];
#pragma unroll
        for (int l = 0; l < kLanes; l++) cnt[l] = 0;
        for (int m = (b - nbv) * blockDim.x + threadIdx.x; m < I.m; m += nbc * blockDim.x) {
            const long long e = (long long)n + m;
            if (acc) {
                L4<T> x[kRowThreads];
                commit(e, x);
            }
            if (chk) {  // CpuSat::CalculateClauses on the accepted state (K2)
                unsigned sat = 0;
#pragma unroll
                for (int q = 0; q < KMAX; q++) {
                    if (EXACT || q < I.k) {
                        Lit<1> w;
                        w.load(I, q * I.mp + m);
                        const bool real = w.var() < (uint32_t)n;
#pragma unroll
                        for (int c = 0; c < kRowThreads; c++) {
                            const L4<T> sv = real ? ld4(A.K2 + (long long)w.var() * kLanes + c * kSub)
                                                  : L4<T>{{T(-1), T(-1), T(-1), T(-1)}};
#pragma unroll
                            for (int l = 0; l < kSub; l++) {
                                const bool t = sv.v[l] > T(0);
                                sat |= ((w.neg() ? !t : t) ? 1u : 0u) << (c * kSub + l);
                            }
                        }
                    }
                }
#pragma unroll
                for (int l = 0; l < kLanes; l++) cnt[l] += ((sat >> l) & 1u) ? 0 : 1;
            }
        }
        if (chk) {
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
            for (int l = 0; l < kLanes; l++) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) cnt[l] += __shfl_xor_sync(0xffffffffu, cnt[l], o);
                if (lane == 0) red[l * 32 + warp] = cnt[l];
            }
            __syncthreads();
            if (threadIdx.x < kLanes && ((chk >> threadIdx.x) & 1u)) {
                int sum = 0;
                for (int i = 0; i < nw; i++) sum += red[threadIdx.x * 32 + i];
                atomicAdd(&A.lanes[threadIdx.x].vcount, sum);
            }
        }
    } else if (chk && A.best_bits) {
        // assignment of lanes at a batch end, public variable order, one word per warp
        const int wpb = blockDim.x >> 5;
        const int nbw = gridDim.x - nbv - nbc;
        for (int wd = (b - nbv - nbc) * wpb + (threadIdx.x >> 5); wd < words; wd += nbw * wpb) {
            const int i = wd * 32 + (threadIdx.x & 31);
            const bool in = i < n;
            const int v = in ? __ldg(I.iperm + i) : 0;
#pragma unroll
            for (int l = 0; l < kLanes; l++) {
                const unsigned bal = __ballot_sync(0xffffffffu, in && A.K2[(long long)v * kLanes + l] > T(0));
                if (((chk >> l) & 1u) && (threadIdx.x & 31) == 0) A.cand_bits[(long long)l * words + wd] = bal;
            }
        }
    }
    if (!last_block(A.tickets + 1, &s_flag)) return;
    if (threadIdx.x < kLanes) {
        LaneState& L = A.lanes[threadIdx.x];
        s_improved[threadIdx.x] = 0;
        if (L.check && L.status == SAT_UNKNOWN) {
            const int viol = L.vcount;
            L.viol = viol;
            if (viol < L.minviol) {
                L.minviol = viol;
                s_improved[threadIdx.x] = A.best_bits != nullptr;
            }
            if (viol == 0) {
                L.status = SAT_SOLUTION_FOUND;
                if (A.stop_on_first) atomicExch(A.inst_solved + A.pidx, 1);
            } else if ((A.deadline && globaltimer_ns() >= *A.deadline) ||
                       (A.stop_on_first && atomicAdd(A.inst_solved + A.pidx, 0) != 0)) {
                L.status = SAT_ODE_INTERRUPTED;
            } else if (!(L.t < A.tmax && L.steps < A.maxsteps)) {
                L.status = L.t >= A.tmax ? SAT_MAXTIME_REACHED : SAT_MAXITER_REACHED;
            }
        }
        L.vcount = 0;
        L.check = 0;
        L.acc = 0;
        if (L.status == SAT_UNKNOWN && L.newstep) {  // next attempt opens a step: k1 evaluation
            L.h = L.hnext;
            L.h0 = L.hnext;
            L.rhs += 1;
        }
        L.newstep = 0;
    }
    __syncthreads();
    for (int l = 0; l < kLanes; l++) {
        if (!s_improved[l]) continue;
        const int u = A.lanes[l].unit;
        uint32_t* dst = A.best_bits + A.unit_bits[u];
        for (int wd = threadIdx.x; wd < words; wd += blockDim.x) dst[wd] = A.cand_bits[(long long)l * words + wd];
    }
    if (threadIdx.x == 0) {
        int act = 0;
        for (int l = 0; l < kLanes; l++) act += A.lanes[l].status == SAT_UNKNOWN;
        *A.active = act;
        A.tickets[1] = 0;
    }
}

// Initial state of a group: public states -> interleaved internal order (a -> log2 a),
// stage-1 spins, sentinel spin row.
template <typename T, bool LOGA>
__global__ void stream_load_kernel(StreamArgs<T> A, const T* __restrict__ states,
                                   const long long* __restrict__ unit_state) {
    const DevInstance& I = A.I;
    const int n = I.n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int l = 0; l < kLanes; l++) {
        const int u = A.lanes[l].unit;
        const T* G = u >= 0 ? states + unit_state[u] : nullptr;
        for (long long i = tid; i < n; i += stride) {
            const int v = __ldg(I.iperm + i);
            const T x = G ? G[i] : T(0);
            A.X[(long long)v * kLanes + l] = x;
            A.SY[(long long)v * kLanes + l] = x;
        }
        for (long long j = tid; j < I.m; j += stride) {
            const long long e = n + __ldg(I.icperm + j);
            const T a = G ? G[n + j] : T(1);
            if constexpr (LOGA) A.X[e * kLanes + l] = log2f(a);
            else A.X[e * kLanes + l] = a;
        }
    }
    if (tid < kLanes) A.SY[(long long)n * kLanes + tid] = T(-1);
}

// Final state of a group back to the public layout, and the lanes' results.
template <typename T, bool LOGA>
__global__ void stream_store_kernel(StreamArgs<T> A, T* __restrict__ states, const long long* __restrict__ unit_state,
                                    UnitResult* __restrict__ results) {
    const DevInstance& I = A.I;
    const int n = I.n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int l = 0; l < kLanes; l++) {
        const LaneState& L = A.lanes[l];
        if (L.unit < 0) continue;
        T* G = states + unit_state[L.unit];
        for (long long i = tid; i < n; i += stride) G[i] = A.X[(long long)__ldg(I.iperm + i) * kLanes + l];
        for (long long j = tid; j < I.m; j += stride) {
            const T v = A.X[(n + (long long)__ldg(I.icperm + j)) * kLanes + l];
            if constexpr (LOGA) G[n + j] = exp2f(v);
            else G[n + j] = v;
        }
        if (tid == 0) {
            UnitResult r;
            r.time = L.t; r.hdid = L.hdid; r.status = L.status; r.steps = L.steps; r.attempts = L.attempts;
            r.rhs = L.rhs; r.viol = L.viol; r.min_viol = L.minviol == INT_MAX ? -1 : L.minviol;
            r.pad0 = r.pad1 = 0;
            results[L.unit] = r;
        }
    }
}

}  // namespace asb
