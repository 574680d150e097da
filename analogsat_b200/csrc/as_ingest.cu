// Device-side ingest: random initial states written straight into HBM, and the DIMACS
// clause body tokenised on the GPU.
//
// Initial states.  The reference fills a state with ISatRandom::GenerateUniform and
// transforms it (ISat::SetRandomState: CpuSat.cpp:123-133 on the host;
// CudaSat1.cu:452-464 with KernelSetInitial1, CudaSatBase.cu:23-55 on the device:
// s = 2u - 1, a = u + 1).  Here the uniforms come from a counter-based generator, so
// every value is a pure function of (seed, draw index) and one thread produces four of
// them from one Philox block, wherever they land.  The generator is Philox4x64-10
// (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011), with the published multipliers and Weyl key increments,
// used the way numpy's Philox bit generator uses it: key (seed, 0), counter starting
// at 1 for the first block, four 64-bit outputs per block in order, and
// u = (x >> 11) * 2^-53.  Trajectories draw consecutively, so a batch of T equal-sized
// trajectories gets exactly numpy.random.Generator(numpy.random.Philox(key=seed))
// .uniform(-1, 1, (T, N)) in its spins.
//
// CNF body.  CnfReader::Read (AnalogSAT/io/CnfReader.cpp:100-127) reads clauses with
// fscanf("%d") until M zeros have been read.  fscanf's grammar makes that a parallel
// problem: every maximal run of digits is one literal, negative when the byte before
// it is '-'; reading fails at the first byte that is neither white space, a digit nor
// a sign, at a sign not followed by a digit, at the end of the file, or (the range
// check that replaces %d's undefined overflow) at a literal whose magnitude exceeds
// 2^31 - 1.  The reader succeeds when the M-th zero comes before the first failure.
// Three kernels: per-tile token and zero counts with the first failure (one 4 KB
// tile per CTA, staged in shared memory with 16-byte loads), one CTA that scans the
// tile counts, and per-tile emission of literals and clause ends at their scanned
// positions.
#include "as_ingest.h"

#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>

namespace asb {
namespace {

constexpr unsigned long long kPhiloxM0 = 0xD2E7470EE14C6C93ull, kPhiloxM1 = 0xCA5A826395121157ull;
constexpr unsigned long long kPhiloxW0 = 0x9E3779B97F4A7C15ull, kPhiloxW1 = 0xBB67AE8584CAA73Bull;

// Philox4x64-10 of the counter (c0, 0, 0, 0) under the key (k0, 0).
__device__ __forceinline__ void philox4x64_10(unsigned long long c0, unsigned long long k0, unsigned long long out[4]) {
    unsigned long long x0 = c0, x1 = 0, x2 = 0, x3 = 0, k1 = 0;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned long long hi0 = __umul64hi(kPhiloxM0, x0), lo0 = kPhiloxM0 * x0;
        const unsigned long long hi1 = __umul64hi(kPhiloxM1, x2), lo1 = kPhiloxM1 * x2;
        x0 = hi1 ^ x1 ^ k0;
        x1 = lo1;
        x2 = hi0 ^ x3 ^ k1;
        x3 = lo0;
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    out[0] = x0;
    out[1] = x1;
    out[2] = x2;
    out[3] = x3;
}

template <typename T> __device__ __forceinline__ T narrow(double v);
template <> __device__ __forceinline__ double narrow<double>(double v) { return v; }
template <> __device__ __forceinline__ float narrow<float>(double v) { return __double2float_rn(v); }

// Last trajectory whose first draw (or fill element) is <= d.
__device__ __forceinline__ int find_traj(const long long* __restrict__ first, int nt, long long d) {
    int lo = 0, hi = nt - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= d) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// One thread per Philox block: draws 4b .. 4b+3 of the stream, written to the
// trajectories (and elements) they belong to.  draw[] holds nt + 1 entries.
template <typename T>
__global__ void __launch_bounds__(256) ic_draw_kernel(T* __restrict__ states, const IcTraj* __restrict__ tr,
                                                      const long long* __restrict__ draw, int nt, long long ndraw,
                                                      unsigned long long seed, int dist) {
    const long long nblk = (ndraw + 3) >> 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nblk; b += stride) {
        unsigned long long r[4];
        philox4x64_10((unsigned long long)b + 1ull, seed, r);
        const long long d0 = b << 2;
        int t = find_traj(draw, nt, d0);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const long long d = d0 + i;
            if (d >= ndraw) break;
            while (draw[t + 1] <= d) t++;
            const long long j = d - draw[t];
            const double u = (double)(r[i] >> 11) * 0x1.0p-53;
            const double v = (dist == kIcSpinUniform || j < tr[t].n) ? __dadd_rn(__dmul_rn(u, 2.0), -1.0)
                                                                    : __dadd_rn(u, 1.0);
            states[tr[t].off + j] = narrow<T>(v);
        }
    }
}

// a_m = a0 for every trajectory (kIcSpinUniform); fill[] holds nt + 1 prefix entries
// of M.  Eight consecutive elements per thread.
template <typename T>
__global__ void __launch_bounds__(256) ic_fill_kernel(T* __restrict__ states, const IcTraj* __restrict__ tr,
                                                      const long long* __restrict__ fill, int nt, long long total, T a0) {
    const long long nchunk = (total + 7) >> 3;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nchunk; c += stride) {
        const long long e0 = c << 3;
        int t = find_traj(fill, nt, e0);
        for (int i = 0; i < 8; i++) {
            const long long e = e0 + i;
            if (e >= total) break;
            while (fill[t + 1] <= e) t++;
            states[tr[t].off + tr[t].n + (e - fill[t])] = a0;
        }
    }
}

int grid_for(long long work, int block) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (work + block - 1) / block;
    return (int)std::max(1ll, std::min(want, (long long)sms * 8));
}

struct Dev {
    void* p = nullptr;
    ~Dev() { if (p) cudaFree(p); }
};

// ---- CNF body ---------------------------------------------------------------------
constexpr int kCnfThreads = 256, kCnfBytes = 16, kCnfTile = kCnfThreads * kCnfBytes;
constexpr unsigned long long kNoFail = ~0ull;

struct CnfHeader {
    unsigned long long fail;  // (position << 1) | range, smallest failure; kNoFail if none
    long long tokens, zeros;  // totals over the body
    long long pos_m;          // position of the M-th zero (-1: not reached)
};

__device__ __forceinline__ bool is_digit(int c) { return c >= '0' && c <= '9'; }
__device__ __forceinline__ bool is_space(int c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// Shared-memory tile: sb[16 + i] = body[base + i]; sb[15] and sb[16 + kCnfTile] are
// the bytes on either side.
struct CnfTile {
    const unsigned char* body;
    long long len, base;
    const unsigned char* sb;
    // Byte at q; -1 outside the body (before it: no digit can precede the body, since
    // the header's last number was read greedily; after it: end of file).
    __device__ __forceinline__ int at(long long q) const {
        if (q < 0 || q >= len) return -1;
        const long long r = q - base;
        if (r >= -1 && r <= kCnfTile) return sb[16 + r];
        return __ldg(body + q);
    }
};

__device__ void stage_tile(const unsigned char* __restrict__ body, long long len, long long base, unsigned char* sb) {
    const int t = threadIdx.x;
    const long long p = base + (long long)t * kCnfBytes;
    if (p + kCnfBytes <= len) {
        *reinterpret_cast<uint4*>(sb + 16 + t * kCnfBytes) = __ldg(reinterpret_cast<const uint4*>(body + p));
    } else {
        for (int i = 0; i < kCnfBytes; i++) sb[16 + t * kCnfBytes + i] = p + i < len ? body[p + i] : 0;
    }
    if (t == 0) sb[15] = base > 0 ? body[base - 1] : ' ';
    if (t == 1) sb[16 + kCnfTile] = base + kCnfTile < len ? body[base + kCnfTile] : 0;
}

// Scans this thread's 16 bytes.  For each literal (run of digits starting here) calls
// emit(position, value, negative, zero); returns the packed counts tokens << 16 | zeros
// and lowers fail to the first failure seen.
template <typename F>
__device__ __forceinline__ int scan_bytes(const CnfTile& T, long long p0, unsigned long long& fail, F&& emit) {
    int tok = 0, zero = 0;
    for (int i = 0; i < kCnfBytes; i++) {
        const long long q = p0 + i;
        if (q >= T.len) break;
        const int c = T.at(q);
        if (is_digit(c)) {
            if (is_digit(T.at(q - 1))) continue;  // inside a literal that started earlier
            long long v = 0;
            bool range = false;
            for (long long r = q;; r++) {
                const int d = T.at(r);
                if (!is_digit(d)) break;
                if (!range) {
                    v = v * 10 + (d - '0');
                    range = v > INT_MAX;
                }
            }
            if (range) fail = min(fail, ((unsigned long long)q << 1) | 1ull);
            emit(q, range ? 0 : (int)v, T.at(q - 1) == '-', v == 0);
            tok++;
            zero += v == 0;
        } else if (c == '+' || c == '-') {
            if (!is_digit(T.at(q + 1))) fail = min(fail, (unsigned long long)q << 1);
        } else if (!is_space(c)) {
            fail = min(fail, (unsigned long long)q << 1);
        }
    }
    return (tok << 16) | zero;
}

__device__ __forceinline__ unsigned long long warp_min64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void __launch_bounds__(kCnfThreads) cnf_count_kernel(const unsigned char* __restrict__ body, long long len,
                                                                int* __restrict__ tile_counts, CnfHeader* hdr) {
    __shared__ __align__(16) unsigned char sb[kCnfTile + 32];
    __shared__ int wsum[kCnfThreads / 32];
    __shared__ unsigned long long wfail[kCnfThreads / 32];
    const long long base = (long long)blockIdx.x * kCnfTile;
    stage_tile(body, len, base, sb);
    __syncthreads();
    const CnfTile T{body, len, base, sb};
    unsigned long long fail = kNoFail;
    int c = scan_bytes(T, base + (long long)threadIdx.x * kCnfBytes, fail, [](long long, int, bool, bool) {});
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    fail = warp_min64(fail);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        wsum[w] = c;
        wfail[w] = fail;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        unsigned long long f = kNoFail;
        for (int i = 0; i < kCnfThreads / 32; i++) {
            s += wsum[i];
            f = min(f, wfail[i]);
        }
        tile_counts[blockIdx.x] = s;
        if (f != kNoFail) atomicMin(&hdr->fail, f);
    }
}

// One CTA: exclusive prefixes of the per-tile token and zero counts, and the totals.
__global__ void __launch_bounds__(1024) cnf_scan_kernel(const int* __restrict__ tile_counts, long long ntiles,
                                                        long long* __restrict__ tok_pre, long long* __restrict__ zero_pre,
                                                        CnfHeader* hdr) {
    __shared__ long long st[1024], sz[1024];
    const int t = threadIdx.x;
    const long long per = (ntiles + 1023) / 1024;
    const long long lo = t * per < ntiles ? t * per : ntiles, hi = lo + per < ntiles ? lo + per : ntiles;
    long long a = 0, z = 0;
    for (long long i = lo; i < hi; i++) {
        a += tile_counts[i] >> 16;
        z += tile_counts[i] & 0xffff;
    }
    st[t] = a;
    sz[t] = z;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // inclusive Hillis-Steele scan
        const long long pa = t >= o ? st[t - o] : 0, pz = t >= o ? sz[t - o] : 0;
        __syncthreads();
        st[t] += pa;
        sz[t] += pz;
        __syncthreads();
    }
    long long ra = st[t] - a, rz = sz[t] - z;
    for (long long i = lo; i < hi; i++) {
        tok_pre[i] = ra;
        zero_pre[i] = rz;
        ra += tile_counts[i] >> 16;
        rz += tile_counts[i] & 0xffff;
    }
    if (t == 1023) {
        hdr->tokens = st[t];
        hdr->zeros = sz[t];
    }
}

// Literal with token index k and zero index z (zeros before it) of clause z goes to
// literals[k - z]; the zero closing clause z records ends[z] = k - z.  Only the
// first m clauses are written.
__global__ void __launch_bounds__(kCnfThreads) cnf_emit_kernel(const unsigned char* __restrict__ body, long long len,
                                                               const long long* __restrict__ tok_pre,
                                                               const long long* __restrict__ zero_pre, long long m,
                                                               int* __restrict__ literals, int* __restrict__ ends,
                                                               CnfHeader* hdr) {
    __shared__ __align__(16) unsigned char sb[kCnfTile + 32];
    __shared__ int wsum[kCnfThreads / 32];
    const long long base = (long long)blockIdx.x * kCnfTile;
    stage_tile(body, len, base, sb);
    __syncthreads();
    const CnfTile T{body, len, base, sb};
    const long long p0 = base + (long long)threadIdx.x * kCnfBytes;
    unsigned long long fail = kNoFail;
    const int c = scan_bytes(T, p0, fail, [](long long, int, bool, bool) {});
    // exclusive block scan of the packed counts
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    int before = 0;
    for (int i = 0; i < w; i++) before += wsum[i];
    const int ex = before + inc - c;
    long long k = tok_pre[blockIdx.x] + (ex >> 16);
    long long z = zero_pre[blockIdx.x] + (ex & 0xffff);
    scan_bytes(T, p0, fail, [&](long long q, int v, bool neg, bool is_zero) {
        if (z < m) {
            if (is_zero) {
                ends[z] = (int)(k - z);
                if (z == m - 1) hdr->pos_m = q;
            } else {
                literals[k - z] = neg ? -v : v;
            }
        }
        z += is_zero;
        k++;
    });
}

}  // namespace

cudaError_t random_states(void* states, bool f64, const std::vector<IcTraj>& traj, unsigned long long seed,
                          int distribution, double a0, cudaStream_t stream) {
    const int nt = (int)traj.size();
    if (nt == 0) return cudaSuccess;
    // prefix tables (with a sentinel) of the draws and of the constant elements
    std::vector<long long> draw(nt + 1, 0), fill(nt + 1, 0);
    for (int t = 0; t < nt; t++) {
        const bool spin_only = distribution == kIcSpinUniform;
        draw[t + 1] = draw[t] + traj[t].n + (spin_only ? 0 : traj[t].m);
        fill[t + 1] = fill[t] + (spin_only ? traj[t].m : 0);
    }
    Dev dt, dd, df;
    const size_t tb = sizeof(IcTraj) * nt, lb = sizeof(long long) * (nt + 1);
    cudaError_t e;
    if ((e = cudaMalloc(&dt.p, tb)) || (e = cudaMalloc(&dd.p, lb)) || (e = cudaMalloc(&df.p, lb))) return e;
    if ((e = cudaMemcpyAsync(dt.p, traj.data(), tb, cudaMemcpyHostToDevice, stream)) ||
        (e = cudaMemcpyAsync(dd.p, draw.data(), lb, cudaMemcpyHostToDevice, stream)) ||
        (e = cudaMemcpyAsync(df.p, fill.data(), lb, cudaMemcpyHostToDevice, stream)))
        return e;
    const long long ndraw = draw[nt];
    const auto* T = static_cast<const IcTraj*>(dt.p);
    const auto* D = static_cast<const long long*>(dd.p);
    const auto* F = static_cast<const long long*>(df.p);
    if (ndraw > 0) {
        const int g = grid_for((ndraw + 3) / 4, 256);
        if (f64) ic_draw_kernel<double><<<g, 256, 0, stream>>>(static_cast<double*>(states), T, D, nt, ndraw, seed, distribution);
        else ic_draw_kernel<float><<<g, 256, 0, stream>>>(static_cast<float*>(states), T, D, nt, ndraw, seed, distribution);
        if ((e = cudaGetLastError())) return e;
    }
    if (fill[nt] > 0) {
        const int g = grid_for((fill[nt] + 7) / 8, 256);
        if (f64) ic_fill_kernel<double><<<g, 256, 0, stream>>>(static_cast<double*>(states), T, F, nt, fill[nt], a0);
        else ic_fill_kernel<float><<<g, 256, 0, stream>>>(static_cast<float*>(states), T, F, nt, fill[nt], (float)a0);
        if ((e = cudaGetLastError())) return e;
    }
    return cudaStreamSynchronize(stream);
}

bool parse_cnf_body(const char* body, size_t len, long long m, std::vector<int32_t>& literals,
                    std::vector<int32_t>& lengths, std::string& msg, cudaError_t& cuda) {
    cuda = cudaSuccess;
    literals.clear();
    lengths.clear();
    msg = "read ok";
    if (m <= 0) return true;
#define AS_ING(call)                                            \
    do {                                                        \
        if ((cuda = (call)) != cudaSuccess) {                   \
            msg = std::string(#call) + ": " + cudaGetErrorString(cuda); \
            return false;                                       \
        }                                                       \
    } while (0)
    cudaStream_t st = nullptr;
    AS_ING(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> st_guard(st, [](cudaStream_t s) { cudaStreamDestroy(s); });
    const long long ntiles = std::max<long long>(1, ((long long)len + kCnfTile - 1) / kCnfTile);
    Dev dbody, dcounts, dtok, dzero, dhdr;
    AS_ING(cudaMalloc(&dbody.p, std::max<size_t>(len, 16)));
    AS_ING(cudaMalloc(&dcounts.p, sizeof(int) * ntiles));
    AS_ING(cudaMalloc(&dtok.p, sizeof(long long) * ntiles));
    AS_ING(cudaMalloc(&dzero.p, sizeof(long long) * ntiles));
    AS_ING(cudaMalloc(&dhdr.p, sizeof(CnfHeader)));
    CnfHeader h{kNoFail, 0, 0, -1};
    AS_ING(cudaMemcpyAsync(dhdr.p, &h, sizeof h, cudaMemcpyHostToDevice, st));
    if (len) AS_ING(cudaMemcpyAsync(dbody.p, body, len, cudaMemcpyHostToDevice, st));
    const auto* B = static_cast<const unsigned char*>(dbody.p);
    auto* H = static_cast<CnfHeader*>(dhdr.p);
    if (len) {
        cnf_count_kernel<<<(unsigned)ntiles, kCnfThreads, 0, st>>>(B, (long long)len, static_cast<int*>(dcounts.p), H);
        AS_ING(cudaGetLastError());
    } else {
        AS_ING(cudaMemsetAsync(dcounts.p, 0, sizeof(int), st));
    }
    cnf_scan_kernel<<<1, 1024, 0, st>>>(static_cast<const int*>(dcounts.p), ntiles, static_cast<long long*>(dtok.p),
                                        static_cast<long long*>(dzero.p), H);
    AS_ING(cudaGetLastError());
    AS_ING(cudaMemcpyAsync(&h, H, sizeof h, cudaMemcpyDeviceToHost, st));
    AS_ING(cudaStreamSynchronize(st));
    auto failure = [&](unsigned long long f) {
        msg = (f != kNoFail && (f & 1ull)) ? "literal out of range" : "expected more literals in file";
        return false;
    };
    if (h.zeros < m) return failure(h.fail);  // the M-th zero is never read
    if (h.tokens - h.zeros > INT_MAX) {
        msg = "too many literals";
        return false;
    }
    Dev dlit, dends;
    AS_ING(cudaMalloc(&dlit.p, sizeof(int) * std::max<long long>(1, h.tokens)));
    AS_ING(cudaMalloc(&dends.p, sizeof(int) * m));
    cnf_emit_kernel<<<(unsigned)ntiles, kCnfThreads, 0, st>>>(B, (long long)len, static_cast<const long long*>(dtok.p),
                                                              static_cast<const long long*>(dzero.p), m,
                                                              static_cast<int*>(dlit.p), static_cast<int*>(dends.p), H);
    AS_ING(cudaGetLastError());
    AS_ING(cudaMemcpyAsync(&h, H, sizeof h, cudaMemcpyDeviceToHost, st));
    std::vector<int32_t> ends(m);
    AS_ING(cudaMemcpyAsync(ends.data(), dends.p, sizeof(int) * m, cudaMemcpyDeviceToHost, st));
    AS_ING(cudaStreamSynchronize(st));
    if (h.pos_m < 0 || (h.fail != kNoFail && (long long)(h.fail >> 1) < h.pos_m)) return failure(h.fail);
    literals.resize(ends[m - 1]);
    if (!literals.empty())
        AS_ING(cudaMemcpyAsync(literals.data(), dlit.p, sizeof(int) * literals.size(), cudaMemcpyDeviceToHost, st));
    AS_ING(cudaStreamSynchronize(st));
#undef AS_ING
    lengths.resize(m);
    for (long long c = 0; c < m; c++) lengths[c] = ends[c] - (c ? ends[c - 1] : 0);
    msg = "read ok";
    return true;
}

}  // namespace asb
