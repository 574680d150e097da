// Discrete adjoint of the RK45 (Cash-Karp) integration: gradients of the final
// potential with respect to the initial state and per-clause weights.
//
// Weighted CTDS (w = 1 is the reference ODE, AnalogSAT/cpu_sat/CpuSat.cpp:199-241):
//   ds_i = sum_m 2 w_m a_m c_mi K_mi K_m,   da_m = a_m K_m^2,
//   L    = V(x(T)) = sum_m w_m a_m(T) K_m(s(T))^2.
// adj_forward_kernel runs the adaptive controller to T (last step clamped to land on
// T) and records the accepted step sizes; adj_backward_kernel integrates the frozen
// step sequence again, checkpointing the state before every step in global memory,
// and runs the adjoint recursion backwards through the steps, recomputing each step's
// stage derivatives from its checkpoint:
//   rho_j   = h (c_j lam + sum_{i>j} b_ij sigma_i)        (dL/dk_j)
//   sigma_j = J(y_j)^T rho_j                              (dL/dy_j)
//   lam    <- lam + sum_j sigma_j ,   g_w += (df/dw)(y_j)^T rho_j.
// J^T u is the RHS's vector-Jacobian product -- the Hessian-vector product of V in the
// spin block -- computed with the same clause-phase / var-phase structure as the RHS:
// per clause in registers (leave-one-out and leave-two-out products), per-literal
// contributions stored into the SELL slots, per-variable row sums.
// Linear a in both FP32 and FP64 (over a short horizon a grows at most by e^T).
#pragma once

#include "as_kernels.cuh"

namespace asb {

struct AdjointParams {
    const DevInstance* inst;
    const int* unit_inst;
    const long long* unit_state;   // element offset of each unit's public x0 / grad_x0
    const long long* unit_wofs;    // offset of each unit's clause weights / grad_w (public order)
    const void* x0;                // public layout, solver precision
    const double* weights;         // per clause, public order (null = all 1)
    double* hs;                    // [unit][max_steps] accepted step sizes
    int* nsteps;                   // [unit] steps to reach t_end (-1: more than max_steps, -2 underflow);
                                   // [num_units], [num_units + 1]: work counters of the two kernels
    void* ckpt;                    // backward: per-unit checkpoint area
    const long long* unit_ckpt;    // backward: element offset of each unit's checkpoints
    double* loss;                  // [unit]
    void* grad_x0;                 // public layout, solver precision
    double* grad_w;                // per clause, public order
    int num_units, max_steps;
    double eps, t_end;
};

// Weighted RHS clause phase: contributions use w a, the returned da = a K^2.
template <typename T, int KMAX, bool EXACT>
__device__ __forceinline__ T wclause_fwd(const DevInstance& I, int m, const T* sy, T* cs, T a, T w, T knorm) {
    Lit<0> L[KMAX];
    T f[KMAX];
    T K = knorm;
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (EXACT || q < I.k) {
            L[q].load(I, q * I.mp + m);
            const T s = sy[L[q].var()];
            f[q] = L[q].neg() ? T(1) + s : T(1) - s;
            K *= f[q];
        }
    }
    const T r2 = T(2) * K * knorm * w * a;
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (EXACT || q < I.k) {
            T prod = T(1);
#pragma unroll
            for (int l = 0; l < KMAX; l++)
                if (l != q && (EXACT || l < I.k)) prod *= f[l];
            const T rr = r2 * prod;
            cs[L[q].slot()] = L[q].neg() ? -rr : rr;
        }
    }
    return a * K * K;
}

// VJP clause phase for clause m at state (spins sy, weight a) with cotangent
// (spins su, weight ua): stores the spin-block contributions into cs, returns the
// a-block entry and adds the w-gradient to *gw.
template <typename T, int KMAX, bool EXACT>
__device__ __forceinline__ T wclause_vjp(const DevInstance& I, int m, const T* sy, const T* su, T* cs, T a,
                                         T ua, T w, T knorm, T* gw) {
    Lit<0> L[KMAX];
    T f[KMAX], u[KMAX], c[KMAX], Kq[KMAX];
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (EXACT || q < I.k) {
            L[q].load(I, q * I.mp + m);
            const T s = sy[L[q].var()];
            c[q] = L[q].neg() ? T(-1) : T(1);
            f[q] = T(1) - c[q] * s;
            u[q] = su[L[q].var()];  // the sentinel's cotangent slot holds 0
        }
    }
    T K = knorm;
#pragma unroll
    for (int q = 0; q < KMAX; q++)
        if (EXACT || q < I.k) K *= f[q];
    T S = T(0);
#pragma unroll
    for (int q = 0; q < KMAX; q++) {
        if (EXACT || q < I.k) {
            T p = knorm;
#pragma unroll
            for (int l = 0; l < KMAX; l++)
                if (l != q && (EXACT || l < I.k)) p *= f[l];
            Kq[q] = p;
            S += u[q] * c[q] * p;
        }
    }
    *gw += T(2) * a * S * K;
#pragma unroll
    for (int r = 0; r < KMAX; r++) {
        if (EXACT || r < I.k) {
            T t = Kq[r] * S;  // sum_q u_q c_q K_q K_r
#pragma unroll
            for (int q = 0; q < KMAX; q++) {
                if (q != r && (EXACT || q < I.k)) {
                    T p = knorm;
#pragma unroll
                    for (int l = 0; l < KMAX; l++)
                        if (l != q && l != r && (EXACT || l < I.k)) p *= f[l];
                    t += u[q] * c[q] * p * K;
                }
            }
            cs[L[r].slot()] = T(-2) * c[r] * (w * a * t + ua * a * K * Kq[r]);
        }
    }
    return T(2) * w * S * K + ua * K * K;
}

// Cash-Karp tableau rows used by the adjoint (b_ij for stage i, c_j).
__device__ __forceinline__ double ck_b(int i, int j) {
    switch (i * 8 + j) {
        case 2 * 8 + 1: return ck::b21;
        case 3 * 8 + 1: return ck::b31;
        case 3 * 8 + 2: return ck::b32;
        case 4 * 8 + 1: return ck::b41;
        case 4 * 8 + 2: return ck::b42;
        case 4 * 8 + 3: return ck::b43;
        case 5 * 8 + 1: return ck::b51;
        case 5 * 8 + 2: return ck::b52;
        case 5 * 8 + 3: return ck::b53;
        case 5 * 8 + 4: return ck::b54;
        case 6 * 8 + 1: return ck::b61;
        case 6 * 8 + 2: return ck::b62;
        case 6 * 8 + 3: return ck::b63;
        case 6 * 8 + 4: return ck::b64;
        case 6 * 8 + 5: return ck::b65;
        default: return 0.0;
    }
}
__device__ __forceinline__ double ck_c(int j) {
    switch (j) {
        case 1: return ck::c1;
        case 3: return ck::c3;
        case 4: return ck::c4;
        case 6: return ck::c6;
        default: return 0.0;
    }
}

// Shared-memory layout (E = n + m, Ep = E rounded to 4):
//   V[0..5]   X, K1..K5      V[6] lam      V[7..11] sigma_2..sigma_6   V[12] sigma sum
//   V[13]     weight w (clause part), V[14] grad w accumulator (clause part)
//   sy, su    spins / spin cotangents of the current stage (n+1 each, sentinel at n)
//   cs        contribution slots (nslots + 1)
__host__ __device__ inline size_t adjoint_smem_values(int n, int m, int nslots) {
    const size_t Ep = (size_t)((n + m + 3) & ~3);
    return 15 * Ep + 2 * (size_t)((n + 1 + 3) & ~3) + (size_t)nslots + 1;
}

template <typename T>
struct AdjSmem {
    T* V[15];
    T *sy, *su, *cs;
    __device__ void init(unsigned char* raw, int n, int m) {
        const int Ep = (n + m + 3) & ~3;
        T* b = reinterpret_cast<T*>(raw);
        for (int i = 0; i < 15; i++) V[i] = b + (size_t)i * Ep;
        sy = b + 15 * (size_t)Ep;
        su = sy + ((n + 1 + 3) & ~3);
        cs = su + ((n + 1 + 3) & ~3);
    }
};

// One weighted RHS evaluation at stage S (1..6) of the step at V[0] with step h,
// output into out (an E-vector in shared memory).
template <typename T, int KMAX, bool EXACT, int S>
__device__ __forceinline__ void adj_rhs(const DevInstance& I, const AdjSmem<T>& A, T h, T knorm, T* out) {
    const int tid = threadIdx.x, nt = blockDim.x, n = I.n;
    T* const* V = A.V;
    for (int v = tid; v < n; v += nt) A.sy[v] = stage_in<S>(V[0][v], V[1][v], V[2][v], V[3][v], V[4][v], V[5][v], h);
    __syncthreads();
    for (int m = tid; m < I.m; m += nt) {
        const int e = n + m;
        const T a = stage_in<S>(V[0][e], V[1][e], V[2][e], V[3][e], V[4][e], V[5][e], h);
        out[e] = wclause_fwd<T, KMAX, EXACT>(I, m, A.sy, A.cs, a, V[13][e], knorm);
    }
    __syncthreads();
    for (int v = tid; v < n; v += nt) out[v] = var_phase<T>(I, v, A.cs);
    __syncthreads();
}

// Stage-input of stage j (runtime j) from the stage vectors in V.
template <typename T>
__device__ __forceinline__ T stage_in_rt(int j, T* const* V, int e, T h) {
    switch (j) {
        case 1: return stage_in<1>(V[0][e], V[1][e], V[2][e], V[3][e], V[4][e], V[5][e], h);
        case 2: return stage_in<2>(V[0][e], V[1][e], V[2][e], V[3][e], V[4][e], V[5][e], h);
        case 3: return stage_in<3>(V[0][e], V[1][e], V[2][e], V[3][e], V[4][e], V[5][e], h);
        case 4: return stage_in<4>(V[0][e], V[1][e], V[2][e], V[3][e], V[4][e], V[5][e], h);
        case 5: return stage_in<5>(V[0][e], V[1][e], V[2][e], V[3][e], V[4][e], V[5][e], h);
        default: return stage_in<6>(V[0][e], V[1][e], V[2][e], V[3][e], V[4][e], V[5][e], h);
    }
}

// rho_j for element e from lam and the stored sigmas.
template <typename T>
__device__ __forceinline__ T adj_rho(int j, T* const* V, int e, T h) {
    T acc = T(ck_c(j)) * V[6][e];
    for (int i = j + 1; i <= 6; i++) acc += T(ck_b(i, j)) * V[5 + i][e];  // sigma_i at V[7 + (i-2)]
    return h * acc;
}

// Loads a public-layout vector (spins permuted to the internal order) into dst.
template <typename T>
__device__ __forceinline__ void load_public(const DevInstance& I, const T* src, T* dst) {
    for (int i = threadIdx.x; i < I.n; i += blockDim.x) dst[__ldg(I.iperm + i)] = src[i];
    for (int j = threadIdx.x; j < I.m; j += blockDim.x) dst[I.n + __ldg(I.icperm + j)] = src[I.n + j];
}

template <typename T>
__device__ __forceinline__ void store_public(const DevInstance& I, const T* src, T* dst) {
    for (int i = threadIdx.x; i < I.n; i += blockDim.x) dst[i] = src[__ldg(I.iperm + i)];
    for (int j = threadIdx.x; j < I.m; j += blockDim.x) dst[I.n + j] = src[I.n + __ldg(I.icperm + j)];
}

template <typename T>
__device__ __forceinline__ void load_weights(const DevInstance& I, const AdjointParams& P, int u, T* w) {
    for (int j = threadIdx.x; j < I.m; j += blockDim.x)
        w[I.n + __ldg(I.icperm + j)] = P.weights ? (T)P.weights[P.unit_wofs[u] + j] : T(1);
}

// Adaptive forward pass to t_end recording the accepted step sizes.
template <typename T, int KMAX, bool EXACT>
__global__ void __launch_bounds__(1024, 1) adj_forward_kernel(AdjointParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_d[36];
    __shared__ int s_unit;
    const int tid = threadIdx.x, nt = blockDim.x;
    while (true) {
        if (tid == 0) s_unit = atomicAdd(P.nsteps + P.num_units, 1);
        __syncthreads();
        const int u = s_unit;
        if (u >= P.num_units) break;
        const DevInstance I = P.inst[P.unit_inst[u]];
        const int n = I.n, E = n + I.m;
        AdjSmem<T> A;
        A.init(smem_raw, n, I.m);
        T* const* V = A.V;
        const T knorm = (T)ldexp(1.0, -I.k);
        load_public<T>(I, reinterpret_cast<const T*>(P.x0) + P.unit_state[u], V[0]);
        load_weights<T>(I, P, u, V[13]);
        for (int j = tid; j <= I.nslots; j += nt) A.cs[j] = T(0);
        if (tid == 0) A.sy[n] = T(-1);
        __syncthreads();
        double t = 0.0, hnext = 1e-9;
        int steps = 0, status = 0;
        double* hs = P.hs + (long long)u * P.max_steps;
        while (t < P.t_end) {
            if (steps >= P.max_steps) { status = -1; break; }
            if (t + hnext > P.t_end) hnext = P.t_end - t;
            adj_rhs<T, KMAX, EXACT, 1>(I, A, T(0), knorm, V[1]);
            const double h0 = hnext;
            double h = hnext;
            bool underflow = false;
            while (true) {
                const T hT = (T)h, h0T = (T)h0;
                adj_rhs<T, KMAX, EXACT, 2>(I, A, hT, knorm, V[2]);
                adj_rhs<T, KMAX, EXACT, 3>(I, A, hT, knorm, V[3]);
                adj_rhs<T, KMAX, EXACT, 4>(I, A, hT, knorm, V[4]);
                adj_rhs<T, KMAX, EXACT, 5>(I, A, hT, knorm, V[5]);
                adj_rhs<T, KMAX, EXACT, 6>(I, A, hT, knorm, V[7]);  // k6 (scratch vector)
                T em = T(0);
                for (int e = tid; e < E; e += nt) {
                    const T x = V[0][e], k1 = V[1][e], k3 = V[3][e], k4 = V[4][e], k5 = V[5][e], k6 = V[7][e];
                    em = fmax(em, rk_err_ratio(x, k1, k3, k4, k5, k6, hT, h0T, false));
                    V[8][e] = rk_new<T>(x, k1, k3, k4, k6, hT);
                }
                const double ermax = block_max_then((double)em, red_d, [&](double emax) {
                    const double e = emax / P.eps;
                    double hn;
                    if (e <= 1.0)
                        hn = e > ck::ERRCON ? ck::SAFETY * h * pow(e, ck::PGROW) : 5.0 * h;
                    else
                        hn = fmax(ck::SAFETY * h * pow(e, ck::PSHRNK), ck::HFACTOR * h);
                    red_d[34] = hn;
                    return e;
                });
                const double hn = red_d[34];
                if (ermax <= 1.0) { hnext = hn; break; }
                h = hn;
                if (t + h == t) { underflow = true; break; }
            }
            if (underflow) { status = -2; break; }
            if (tid == 0) hs[steps] = h;
            steps++;
            t += h;
            for (int e = tid; e < E; e += nt) V[0][e] = V[8][e];
            __syncthreads();
        }
        if (tid == 0) P.nsteps[u] = status ? status : steps;
        __syncthreads();
    }
}

// Fixed-step forward with checkpoints, then the adjoint recursion.
template <typename T, int KMAX, bool EXACT>
__global__ void __launch_bounds__(1024, 1) adj_backward_kernel(AdjointParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_d[36];
    __shared__ int s_unit;
    const int tid = threadIdx.x, nt = blockDim.x;
    while (true) {
        if (tid == 0) s_unit = atomicAdd(P.nsteps + P.num_units + 1, 1);
        __syncthreads();
        const int u = s_unit;
        if (u >= P.num_units) break;
        const int ns = P.nsteps[u];
        const DevInstance I = P.inst[P.unit_inst[u]];
        const int n = I.n, E = n + I.m;
        AdjSmem<T> A;
        A.init(smem_raw, n, I.m);
        T* const* V = A.V;
        const T knorm = (T)ldexp(1.0, -I.k);
        const double* hs = P.hs + (long long)u * P.max_steps;
        T* ck = reinterpret_cast<T*>(P.ckpt) + P.unit_ckpt[u];
        load_public<T>(I, reinterpret_cast<const T*>(P.x0) + P.unit_state[u], V[0]);
        load_weights<T>(I, P, u, V[13]);
        for (int j = tid; j <= I.nslots; j += nt) A.cs[j] = T(0);
        if (tid == 0) { A.sy[n] = T(-1); A.su[n] = T(0); }
        __syncthreads();
        // forward through the frozen step sequence, checkpoint before every step
        for (int s = 0; s < ns; s++) {
            const T h = (T)hs[s];
            for (int e = tid; e < E; e += nt) ck[(long long)s * E + e] = V[0][e];
            adj_rhs<T, KMAX, EXACT, 1>(I, A, h, knorm, V[1]);
            adj_rhs<T, KMAX, EXACT, 2>(I, A, h, knorm, V[2]);
            adj_rhs<T, KMAX, EXACT, 3>(I, A, h, knorm, V[3]);
            adj_rhs<T, KMAX, EXACT, 4>(I, A, h, knorm, V[4]);
            adj_rhs<T, KMAX, EXACT, 5>(I, A, h, knorm, V[5]);
            adj_rhs<T, KMAX, EXACT, 6>(I, A, h, knorm, V[7]);
            for (int e = tid; e < E; e += nt)
                V[0][e] = rk_new<T>(V[0][e], V[1][e], V[3][e], V[4][e], V[7][e], h);
            __syncthreads();
        }
        // dL/dx(T) = (-ds/dt(x_T), w K^2), dL/dw = a K^2, L = sum w a K^2
        adj_rhs<T, KMAX, EXACT, 1>(I, A, T(0), knorm, V[1]);
        double lsum = 0.0;
        for (int v = tid; v < n; v += nt) V[6][v] = -V[1][v];
        for (int m = tid; m < I.m; m += nt) {
            const int e = n + m;
            const T a = V[0][e], K2 = a != T(0) ? V[1][e] / a : T(0);
            V[6][e] = V[13][e] * K2;
            V[14][e] = a * K2;
            lsum += (double)(V[13][e] * a * K2);
        }
        // loss = sum of the per-thread terms (warp shuffles, one slot per warp)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        __syncthreads();
        if ((tid & 31) == 0) red_d[tid >> 5] = lsum;
        __syncthreads();
        if (tid == 0) {
            double sacc = 0.0;
            for (int w = 0; w < (nt >> 5); w++) sacc += red_d[w];
            P.loss[u] = sacc;
        }
        __syncthreads();
        // backward over the steps
        for (int s = ns - 1; s >= 0; s--) {
            const T h = (T)hs[s];
            for (int e = tid; e < E; e += nt) V[0][e] = ck[(long long)s * E + e];
            __syncthreads();
            adj_rhs<T, KMAX, EXACT, 1>(I, A, h, knorm, V[1]);
            adj_rhs<T, KMAX, EXACT, 2>(I, A, h, knorm, V[2]);
            adj_rhs<T, KMAX, EXACT, 3>(I, A, h, knorm, V[3]);
            adj_rhs<T, KMAX, EXACT, 4>(I, A, h, knorm, V[4]);
            adj_rhs<T, KMAX, EXACT, 5>(I, A, h, knorm, V[5]);
            for (int e = tid; e < E; e += nt) V[12][e] = T(0);
            for (int j = 6; j >= 1; j--) {
                // spins and spin cotangents of stage j
                for (int v = tid; v < n; v += nt) {
                    A.sy[v] = stage_in_rt<T>(j, V, v, h);
                    A.su[v] = adj_rho<T>(j, V, v, h);
                }
                __syncthreads();
                for (int m = tid; m < I.m; m += nt) {
                    const int e = n + m;
                    const T a = stage_in_rt<T>(j, V, e, h);
                    const T ua = adj_rho<T>(j, V, e, h);
                    T gw = T(0);
                    const T sg = wclause_vjp<T, KMAX, EXACT>(I, m, A.sy, A.su, A.cs, a, ua, V[13][e], knorm, &gw);
                    V[14][e] += gw;
                    V[12][e] += sg;
                    if (j >= 2) V[5 + j][e] = sg;
                }
                __syncthreads();
                for (int v = tid; v < n; v += nt) {
                    const T sg = var_phase<T>(I, v, A.cs);
                    V[12][v] += sg;
                    if (j >= 2) V[5 + j][v] = sg;
                }
                __syncthreads();
            }
            for (int e = tid; e < E; e += nt) V[6][e] += V[12][e];
            __syncthreads();
        }
        store_public<T>(I, V[6], reinterpret_cast<T*>(P.grad_x0) + P.unit_state[u]);
        for (int j = tid; j < I.m; j += nt)
            P.grad_w[P.unit_wofs[u] + j] = (double)V[14][n + __ldg(I.icperm + j)];
        __syncthreads();
    }
}

}  // namespace asb
