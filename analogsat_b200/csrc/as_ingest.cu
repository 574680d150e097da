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

// Per trajectory on the device: state offset, first draw of the stream, N and M.
struct IcRow {
    long long off, draw;
    int n, m;
};

constexpr int kIcChunk = 1024;    // draws per CTA of ic_draw_kernel
constexpr int kFillChunk = 8192;  // constant elements per CTA of ic_fill_kernel

// Grid (chunks, trajectories): CTA (x, y) takes draws [x * kIcChunk, +kIcChunk) of
// trajectories y, y + gridDim.y, ...  It computes the Philox blocks covering them (one
// per thread), stages the values in shared memory and stores them with consecutive
// threads on consecutive elements.
template <typename T>
__global__ void __launch_bounds__(256) ic_draw_kernel(T* __restrict__ states, const IcRow* __restrict__ rows, int nt,
                                                      unsigned long long seed, int dist) {
    __shared__ T vals[kIcChunk];
    for (int t = blockIdx.y; t < nt; t += gridDim.y) {
        const IcRow R = rows[t];
        const long long j0 = (long long)blockIdx.x * kIcChunk;
        const long long ndraw = R.n + (dist == kIcSpinUniform ? 0 : (long long)R.m);
        if (j0 >= ndraw) continue;  // uniform across the CTA
        const int cnt = (int)min((long long)kIcChunk, ndraw - j0);
        const long long d0 = R.draw + j0;
        const long long b0 = d0 >> 2;
        const int nb = (int)(((d0 + cnt - 1) >> 2) - b0 + 1);
        for (int i = threadIdx.x; i < nb; i += blockDim.x) {
            unsigned long long r[4];
            philox4x64_10((unsigned long long)(b0 + i) + 1ull, seed, r);
            const long long e0 = ((b0 + i) << 2) - d0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const long long e = e0 + k;
                if (e < 0 || e >= cnt) continue;
                const double u = (double)(r[k] >> 11) * 0x1.0p-53;
                const bool spin = dist == kIcSpinUniform || j0 + e < R.n;
                vals[e] = narrow<T>(spin ? __dadd_rn(__dmul_rn(u, 2.0), -1.0) : __dadd_rn(u, 1.0));
            }
        }
        __syncthreads();
        T* dst = states + R.off + j0;
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) dst[e] = vals[e];
        __syncthreads();
    }
}

// a_m = a0 (kIcSpinUniform).  Grid (chunks, trajectories): CTA (x, y) fills weights
// [x * kFillChunk, +kFillChunk) of trajectories y, y + gridDim.y, ... with 16-byte
// stores between a scalar head and tail; the next trajectory's row is loaded before
// the current stores are issued.
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static __device__ float4 splat(float v) { return make_float4(v, v, v, v); } };
template <> struct Vec16<double> { using type = double2; static __device__ double2 splat(double v) { return make_double2(v, v); } };

template <typename T>
__global__ void __launch_bounds__(256) ic_fill_kernel(T* __restrict__ states, const IcRow* __restrict__ rows, int nt,
                                                      T a0) {
    using V = typename Vec16<T>::type;
    constexpr int kPer = 16 / sizeof(T);
    const V v = Vec16<T>::splat(a0);
    int t = blockIdx.y;
    if (t >= nt) return;
    IcRow R = rows[t];
    for (; t < nt; t += gridDim.y) {
        const IcRow Rn = t + (int)gridDim.y < nt ? rows[t + gridDim.y] : R;
        const long long j0 = (long long)blockIdx.x * kFillChunk;
        if (j0 < R.m) {
            const int cnt = (int)min((long long)kFillChunk, (long long)R.m - j0);
            T* dst = states + R.off + R.n + j0;
            const int head = min(cnt, (int)(((16u - ((unsigned)(uintptr_t)dst & 15u)) & 15u) / sizeof(T)));
            if ((int)threadIdx.x < head) dst[threadIdx.x] = a0;
            const int nvec = (cnt - head) / kPer;
            V* vd = reinterpret_cast<V*>(dst + head);
            for (int i = threadIdx.x; i < nvec; i += blockDim.x) vd[i] = v;
            const int done = head + nvec * kPer;
            if ((int)threadIdx.x < cnt - done) dst[done + threadIdx.x] = a0;
        }
        R = Rn;
    }
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

// Byte classes of four bytes at once: each returns 0x80 in the bytes where the class
// holds (C locale: white space is ' ' and '\t'..'\r').
__device__ __forceinline__ unsigned cls_digit(unsigned w) { return __vcmpltu4(__vsub4(w, 0x30303030u), 0x0a0a0a0au) & 0x80808080u; }
__device__ __forceinline__ unsigned cls_nonzero(unsigned w) { return __vcmpltu4(__vsub4(w, 0x31313131u), 0x09090909u) & 0x80808080u; }
__device__ __forceinline__ unsigned cls_space(unsigned w) {
    return (__vcmpeq4(w, 0x20202020u) | __vcmpltu4(__vsub4(w, 0x09090909u), 0x05050505u)) & 0x80808080u;
}
__device__ __forceinline__ unsigned cls_minus(unsigned w) { return __vcmpeq4(w, 0x2d2d2d2du) & 0x80808080u; }
__device__ __forceinline__ unsigned cls_sign(unsigned w) { return (__vcmpeq4(w, 0x2b2b2b2bu) & 0x80808080u) | cls_minus(w); }
// 0x80 flags of four bytes -> bits 0..3 (byte 0 -> bit 0)
__device__ __forceinline__ unsigned pack4(unsigned f) { return ((f >> 7) * 0x10204080u) >> 28; }

template <unsigned (*F)(unsigned)>
__device__ __forceinline__ unsigned mask16(const uint4& v) {
    return pack4(F(v.x)) | pack4(F(v.y)) << 4 | pack4(F(v.z)) << 8 | pack4(F(v.w)) << 12;
}

// Byte i (0..31) of a thread's own 16 bytes followed by the next 16.
__device__ __forceinline__ int byte_at(const uint4& a, const uint4& b, int i) {
    const int k = i >> 2;
    unsigned w = a.x;
    w = k == 1 ? a.y : w;
    w = k == 2 ? a.z : w;
    w = k == 3 ? a.w : w;
    w = k == 4 ? b.x : w;
    w = k == 5 ? b.y : w;
    w = k == 6 ? b.z : w;
    w = k == 7 ? b.w : w;
    return (w >> ((i & 3) * 8)) & 0xff;
}

// Shared-memory tile: sb[16 + i] = body[base + i] for i < kCnfTile + 16 (the tile and
// the 16 bytes after it); sb[15] = the byte before (' ' for the first tile).
__device__ void stage_tile(const unsigned char* __restrict__ body, long long len, long long base, unsigned char* sb) {
    for (int c = threadIdx.x; c < kCnfTile / 16 + 1; c += blockDim.x) {
        const long long p = base + 16ll * c;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (p + 16 <= len) {
            v = __ldg(reinterpret_cast<const uint4*>(body + p));
        } else if (p < len) {
            unsigned char t[16];
            for (int i = 0; i < 16; i++) t[i] = p + i < len ? body[p + i] : 0;
            memcpy(&v, t, 16);
        }
        *reinterpret_cast<uint4*>(sb + 16 + 16 * c) = v;
    }
    if (threadIdx.x == 0) sb[15] = base > 0 ? body[base - 1] : ' ';
}

// A literal (maximal run of digits) starting at byte q of the body, scanned in global
// memory: its value (saturated), whether it is zero and whether it is out of range.
__device__ void scan_long(const unsigned char* __restrict__ body, long long len, long long q, long long& v, bool& range) {
    v = 0;
    range = false;
    for (long long r = q; r < len; r++) {
        const int d = body[r];
        if (d < '0' || d > '9') break;
        if (!range) {
            v = v * 10 + (d - '0');
            range = v > INT_MAX;
        }
    }
}

// Byte-class masks of one thread's 16 bytes at body position p0 (own: those bytes,
// next: the 16 after them, prev: the byte before): bit i of dig / nz is byte i of the
// 32 (digit / digit 1-9), of mn and starts byte i of the own 16 ('-' / first digit of
// a literal).  Lowers fail to the first malformed byte among the own 16.
struct ByteMasks {
    unsigned dig, nz, mn, starts;
    bool prev_mn;
};

__device__ __forceinline__ ByteMasks byte_masks(long long len, long long p0, const uint4& own, const uint4& next,
                                                int prev, unsigned long long& fail) {
    ByteMasks k{0u, 0u, 0u, 0u, false};
    const long long avail = len - p0;
    if (avail <= 0) return k;
    const unsigned valid = avail >= 32 ? 0xffffffffu : (1u << avail) - 1u;
    k.dig = (mask16<cls_digit>(own) | mask16<cls_digit>(next) << 16) & valid;
    k.nz = (mask16<cls_nonzero>(own) | mask16<cls_nonzero>(next) << 16) & valid;
    const unsigned sp = mask16<cls_space>(own) & valid;
    const unsigned sg = mask16<cls_sign>(own) & valid;
    k.mn = mask16<cls_minus>(own) & valid;
    const unsigned prev_dig = (prev >= '0' && prev <= '9') ? 1u : 0u;
    k.prev_mn = prev == '-';
    // failures: a byte of no class, a sign without a digit right after it
    const unsigned bad = ((~(k.dig | sp | sg) & valid) | (sg & ~(k.dig >> 1))) & 0xffffu;
    if (bad) fail = min(fail, (unsigned long long)(p0 + __ffs(bad) - 1) << 1);
    k.starts = k.dig & ~((k.dig << 1) | prev_dig) & 0xffffu;
    return k;
}

// Walks the literals starting in these 16 bytes: emit(position, value, negative,
// zero) for each (value only when VALUES); returns the packed counts tokens << 16 |
// zeros and lowers fail at an out-of-range literal.
template <bool VALUES, typename F>
__device__ __forceinline__ int walk_literals(const unsigned char* __restrict__ body, long long len, long long p0,
                                             const uint4& own, const uint4& next, const ByteMasks& k,
                                             unsigned long long& fail, F&& emit) {
    unsigned starts = k.starts;
    int tok = 0, zero = 0;
    while (starts) {
        const int s = __ffs(starts) - 1;
        starts &= starts - 1;
        const unsigned rest = ~(k.dig >> s);  // bit j: byte s + j is not a digit
        const int e = rest ? s + __ffs(rest) - 1 : 32;
        long long v = 0;
        bool range = false, is_zero;
        if (e >= 32) {  // the run may continue past the 32 bytes in registers
            scan_long(body, len, p0 + s, v, range);
            is_zero = v == 0;
        } else {
            const unsigned run = (1u << (e - s)) - 1u;
            const unsigned nzr = (k.nz >> s) & run;
            is_zero = nzr == 0;
            if (!is_zero) {
                const int sig = e - s - (__ffs(nzr) - 1);  // digits after the leading zeros
                if (sig > 10) {
                    range = true;
                } else if (VALUES || sig == 10) {  // ten digits may still exceed 2^31 - 1
                    for (int i = e - sig; i < e; i++) v = v * 10 + (byte_at(own, next, i) - '0');
                    range = v > INT_MAX;
                }
            }
        }
        if (range) fail = min(fail, ((unsigned long long)(p0 + s) << 1) | 1ull);
        const bool neg = s ? ((k.mn >> (s - 1)) & 1u) : k.prev_mn;
        emit(p0 + s, range ? 0 : (int)v, neg, is_zero);
        tok++;
        zero += is_zero;
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
    const int tid = threadIdx.x;
    const uint4 own = *reinterpret_cast<const uint4*>(sb + 16 + kCnfBytes * tid);
    const uint4 next = *reinterpret_cast<const uint4*>(sb + 32 + kCnfBytes * tid);
    unsigned long long fail = kNoFail;
    const long long p0 = base + (long long)kCnfBytes * tid;
    const ByteMasks k = byte_masks(len, p0, own, next, sb[15 + kCnfBytes * tid], fail);
    int c = walk_literals<false>(body, len, p0, own, next, k, fail, [](long long, int, bool, bool) {});
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
    const int tid = threadIdx.x;
    const uint4 own = *reinterpret_cast<const uint4*>(sb + 16 + kCnfBytes * tid);
    const uint4 next = *reinterpret_cast<const uint4*>(sb + 32 + kCnfBytes * tid);
    const int prev = sb[15 + kCnfBytes * tid];
    const long long p0 = base + (long long)kCnfBytes * tid;
    unsigned long long fail = kNoFail;
    const ByteMasks bm = byte_masks(len, p0, own, next, prev, fail);
    const int c = walk_literals<false>(body, len, p0, own, next, bm, fail, [](long long, int, bool, bool) {});
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
    walk_literals<true>(body, len, p0, own, next, bm, fail, [&](long long q, int v, bool neg, bool is_zero) {
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
    // per trajectory: offset, first draw, N, M; the longest draw and weight runs
    std::vector<IcRow> rows(nt);
    long long draw = 0, max_draw = 0, max_m = 0;
    const bool spin_only = distribution == kIcSpinUniform;
    for (int t = 0; t < nt; t++) {
        const long long nd = traj[t].n + (spin_only ? 0 : (long long)traj[t].m);
        rows[t] = IcRow{traj[t].off, draw, traj[t].n, traj[t].m};
        draw += nd;
        max_draw = std::max(max_draw, nd);
        max_m = std::max(max_m, (long long)traj[t].m);
    }
    Dev dr;
    const size_t rb = sizeof(IcRow) * nt;
    cudaError_t e;
    if ((e = cudaMalloc(&dr.p, rb))) return e;
    if ((e = cudaMemcpyAsync(dr.p, rows.data(), rb, cudaMemcpyHostToDevice, stream))) return e;
    const auto* R = static_cast<const IcRow*>(dr.p);
    int dev = 0, sms = 148;
    if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
    // rows of trajectories per grid: about 16 CTAs per SM, so that a CTA takes several
    // trajectories and the load of the next one's row overlaps the current stores
    auto rows_for = [&](long long gx) {
        return (unsigned)std::max(1ll, std::min<long long>({(long long)nt, 65535ll, 16ll * sms / gx}));
    };
    if (max_draw > 0) {
        const long long gx = (max_draw + kIcChunk - 1) / kIcChunk;
        const dim3 g((unsigned)gx, rows_for(gx));
        if (f64) ic_draw_kernel<double><<<g, 256, 0, stream>>>(static_cast<double*>(states), R, nt, seed, distribution);
        else ic_draw_kernel<float><<<g, 256, 0, stream>>>(static_cast<float*>(states), R, nt, seed, distribution);
        if ((e = cudaGetLastError())) return e;
    }
    if (spin_only && max_m > 0) {
        const long long gx = (max_m + kFillChunk - 1) / kFillChunk;
        const dim3 g((unsigned)gx, rows_for(gx));
        if (f64) ic_fill_kernel<double><<<g, 256, 0, stream>>>(static_cast<double*>(states), R, nt, a0);
        else ic_fill_kernel<float><<<g, 256, 0, stream>>>(static_cast<float*>(states), R, nt, (float)a0);
        if ((e = cudaGetLastError())) return e;
    }
    return cudaStreamSynchronize(stream);
}

bool parse_cnf_body(std::FILE* f, size_t len, long long m, std::vector<int32_t>& literals,
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
    {
        // the body crosses in kStage pieces through two pinned buffers, so that reading
        // the next piece from the file overlaps the copy of the previous one
        constexpr size_t kStage = 4u << 20;
        char* stage = nullptr;
        AS_ING(cudaHostAlloc(reinterpret_cast<void**>(&stage), 2 * kStage, cudaHostAllocDefault));
        std::unique_ptr<char, cudaError_t (*)(void*)> stage_guard(stage, cudaFreeHost);
        cudaEvent_t ev[2] = {nullptr, nullptr};
        AS_ING(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
        std::unique_ptr<CUevent_st, cudaError_t (*)(cudaEvent_t)> ev0_guard(ev[0], cudaEventDestroy);
        AS_ING(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
        std::unique_ptr<CUevent_st, cudaError_t (*)(cudaEvent_t)> ev1_guard(ev[1], cudaEventDestroy);
        size_t off = 0;
        for (int i = 0; off < len; i++) {
            const size_t c = std::min(kStage, len - off);
            char* hbuf = stage + (i & 1) * kStage;
            if (i >= 2) AS_ING(cudaEventSynchronize(ev[i & 1]));  // its previous copy is done
            if (std::fread(hbuf, 1, c, f) != c) {
                cudaStreamSynchronize(st);
                msg = "read failed";
                return false;
            }
            AS_ING(cudaMemcpyAsync(static_cast<char*>(dbody.p) + off, hbuf, c, cudaMemcpyHostToDevice, st));
            AS_ING(cudaEventRecord(ev[i & 1], st));
            off += c;
        }
        AS_ING(cudaStreamSynchronize(st));  // before the staging buffers go
    }
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
