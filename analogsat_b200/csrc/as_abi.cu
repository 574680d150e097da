// C ABI of the AnalogSAT B200 solver (declarations and reference mapping in
// include/analogsat_b200.h).  Host logic: problem handles, device packing,
// launch-shape selection, the persistent solve launch (captured in a CUDA graph),
// and the batched RHS / clause-check primitives.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <ctime>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstddef>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/analogsat_b200.h"
#include "as_ingest.h"
#include "as_fast.cuh"
#include "as_kernels.cuh"
#include "as_problem.h"
#include "as_stream.cuh"

using namespace asb;

// layout index of the pair RHS kernel's packing (after the two precisions)
constexpr int kLayoutPair = AS_LAYOUT_F32_PAIR;

// The plain CTDS right-hand side (CpuSat with b = 0): what every kernel supports.
bool standard_model(const PackedProblem& q) { return !q.tanh && !(q.b > 0.0); }

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define AS_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(AS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t b) {
        if (b <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(b, 16));
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Device copy of one or more packed instances in a single pool.
struct DevicePool {
    int device = -1;
    DevBuf lit, litw, slotw, srow, perm, iperm, icperm, cperm, inst, flit;
    DevBuf plit, pc0, psrow, pcnt, picperm;  // clause-parts layouts (lean global-rows form)
    std::vector<DevInstance> host_inst;

    template <typename V>
    static int put(const DevBuf& buf, size_t off, const V& v) {
        if (!v.empty())
            AS_CUDA(cudaMemcpy(static_cast<char*>(buf.p) + off * 4, v.data(), v.size() * 4,
                               cudaMemcpyHostToDevice));
        return AS_OK;
    }

    int upload(const std::vector<const PackedProblem*>& pk, int dev,
               const std::vector<PartLayout>* parts = nullptr) {
        size_t nl = 0, nw = 0, nr = 0, np = 0, nc = 0;
        for (auto* q : pk) {
            nl += q->lit.size();
            nw += q->litw.size();
            nr += q->srow.size();
            np += q->perm.size();
            nc += q->icperm.size();
        }
        AS_CUDA(lit.alloc(std::max<size_t>(nl, 1) * 4));
        AS_CUDA(litw.alloc(std::max<size_t>(nw, 1) * 4));
        AS_CUDA(slotw.alloc(std::max<size_t>(nw, 1) * 4));
        AS_CUDA(srow.alloc(std::max<size_t>(nr, 1) * 4));
        AS_CUDA(perm.alloc(std::max<size_t>(np, 1) * 4));
        AS_CUDA(iperm.alloc(std::max<size_t>(np, 1) * 4));
        AS_CUDA(icperm.alloc(std::max<size_t>(nc, 1) * 4));
        AS_CUDA(cperm.alloc(std::max<size_t>(nc, 1) * 4));
        AS_CUDA(inst.alloc(sizeof(DevInstance) * std::max<size_t>(pk.size(), 1)));
        // literal words with shared-memory addressing for the lean FP32 solver, for the
        // instances that fit (bits 0-13 spin byte offset, 14-30 slot index, 31 sign),
        // blocked by 32 clauses (lean_word_index)
        std::vector<uint32_t> fw;
        std::vector<long long> fw_off;
        for (auto* q : pk) {
            const FastLayout L = fast_layout(q->n, q->m, q->nslots);
            if (!q->compact || (q->k != 3 && q->k != 4) || !L.ok) {
                fw_off.push_back(-1);
                continue;
            }
            const size_t f0 = fw.size();
            fw_off.push_back((long long)f0);
            fw.resize(f0 + lean_words(q->m, q->k), 0u);
            for (int c = 0; c < q->m; c++)
                for (int qq = 0; qq < q->k; qq++) {
                    const uint32_t w = q->lit[(size_t)qq * q->mp + c];
                    const uint32_t var = (w >> 16) & 0x7fffu, slot = w & 0xffffu;
                    // a negated literal addresses the negated spin copy (neg_spin_base)
                    const uint32_t so = 4u * var + ((w & 0x80000000u) ? 4u * (uint32_t)neg_spin_base(q->n) : 0u);
                    fw[f0 + lean_word_index(c, qq, q->k)] = (w & 0x80000000u) | (slot << 14) | so;
                }
        }
        AS_CUDA(flit.alloc(std::max<size_t>(fw.size(), 1) * 4));
        if (!fw.empty()) AS_CUDA(cudaMemcpy(flit.p, fw.data(), fw.size() * 4, cudaMemcpyHostToDevice));
        // clause parts, concatenated over the problems that have them
        std::vector<uint32_t> pw;
        std::vector<int32_t> pc, ps, pi;
        std::vector<uint16_t> pn;
        std::vector<std::array<size_t, 5>> poff(pk.size(), std::array<size_t, 5>{0, 0, 0, 0, 0});
        if (parts)
            for (size_t i = 0; i < pk.size() && i < parts->size(); i++) {
                const PartLayout& L = (*parts)[i];
                if (L.nparts < 1) continue;
                poff[i] = {pw.size(), pc.size(), ps.size(), pn.size(), pi.size()};
                const size_t w0 = pw.size();  // clause-major words, blocked by 32 clauses
                pw.resize(w0 + lean_words(pk[i]->m, pk[i]->k), 0u);
                for (int c = 0; c < pk[i]->m; c++)
                    for (int qq = 0; qq < pk[i]->k; qq++)
                        pw[w0 + lean_word_index(c, qq, pk[i]->k)] = L.words[(size_t)c * pk[i]->k + qq];
                pc.insert(pc.end(), L.c0.begin(), L.c0.end());
                ps.insert(ps.end(), L.srow.begin(), L.srow.end());
                pn.insert(pn.end(), L.cnt.begin(), L.cnt.end());
                pi.insert(pi.end(), L.icperm.begin(), L.icperm.end());
            }
        AS_CUDA(plit.alloc(std::max<size_t>(pw.size(), 1) * 4));
        AS_CUDA(pc0.alloc(std::max<size_t>(pc.size(), 1) * 4));
        AS_CUDA(psrow.alloc(std::max<size_t>(ps.size(), 1) * 4));
        AS_CUDA(pcnt.alloc(std::max<size_t>(pn.size(), 1) * 2));
        AS_CUDA(picperm.alloc(std::max<size_t>(pi.size(), 1) * 4));
        if (!pw.empty()) {
            AS_CUDA(cudaMemcpy(plit.p, pw.data(), pw.size() * 4, cudaMemcpyHostToDevice));
            AS_CUDA(cudaMemcpy(pc0.p, pc.data(), pc.size() * 4, cudaMemcpyHostToDevice));
            AS_CUDA(cudaMemcpy(psrow.p, ps.data(), ps.size() * 4, cudaMemcpyHostToDevice));
            AS_CUDA(cudaMemcpy(pcnt.p, pn.data(), pn.size() * 2, cudaMemcpyHostToDevice));
            AS_CUDA(cudaMemcpy(picperm.p, pi.data(), pi.size() * 4, cudaMemcpyHostToDevice));
        }
        host_inst.clear();
        size_t ol = 0, ow = 0, orr = 0, op = 0, oc = 0;
        for (auto* q : pk) {
            DevInstance d;
            d.n = q->n; d.m = q->m; d.k = q->k; d.mp = q->mp; d.nslices = q->nslices;
            d.nslots = q->nslots;
            d.tanh = q->tanh;
            d.q = q->q;
            d.b = q->b;
            d.lit = q->lit.empty() ? nullptr : lit.as<uint32_t>() + ol;
            d.litw = litw.as<uint32_t>() + ow;
            d.slotw = slotw.as<uint32_t>() + ow;
            d.srow = srow.as<int32_t>() + orr;
            d.perm = perm.as<int32_t>() + op;
            d.iperm = iperm.as<int32_t>() + op;
            d.icperm = icperm.as<int32_t>() + oc;
            d.cperm = cperm.as<int32_t>() + oc;
            {
                const FastLayout L = fast_layout(q->n, q->m, q->nslots);
                const long long fo = fw_off[host_inst.size()];
                d.flit = fo >= 0 ? flit.as<uint32_t>() + fo : nullptr;
                d.cs_off = L.cs_off;
                d.rows_off = L.rows_off;
                d.cs_off_g = L.cs_off_g;
                const size_t i = host_inst.size();
                const PartLayout* PL = parts && i < parts->size() ? &(*parts)[i] : nullptr;
                d.nparts = PL ? PL->nparts : 0;
                d.part_slots = PL ? PL->max_slots : 0;
                d.plit = d.nparts ? plit.as<uint32_t>() + poff[i][0] : nullptr;
                d.part_c0 = d.nparts ? pc0.as<int32_t>() + poff[i][1] : nullptr;
                d.part_srow = d.nparts ? psrow.as<int32_t>() + poff[i][2] : nullptr;
                d.part_cnt = d.nparts ? pcnt.as<uint16_t>() + poff[i][3] : nullptr;
                d.picperm = d.nparts ? picperm.as<int32_t>() + poff[i][4] : nullptr;
            }
            int r;
            if ((r = put(lit, ol, q->lit)) || (r = put(litw, ow, q->litw)) || (r = put(slotw, ow, q->slotw)) ||
                (r = put(srow, orr, q->srow)) || (r = put(perm, op, q->perm)) ||
                (r = put(iperm, op, q->iperm)) || (r = put(icperm, oc, q->icperm)) ||
                (r = put(cperm, oc, q->cperm)))
                return r;
            ol += q->lit.size();
            ow += q->litw.size();
            orr += q->srow.size();
            op += q->perm.size();
            oc += q->icperm.size();
            host_inst.push_back(d);
        }
        AS_CUDA(cudaMemcpy(inst.p, host_inst.data(), sizeof(DevInstance) * host_inst.size(),
                           cudaMemcpyHostToDevice));
        device = dev;
        return AS_OK;
    }
};

int current_device(int requested, int* out) {
    if (requested >= 0) {
        AS_CUDA(cudaSetDevice(requested));
        *out = requested;
        return AS_OK;
    }
    AS_CUDA(cudaGetDevice(out));
    return AS_OK;
}

// ---------------------------------------------------------------------------
// compiled launch shapes of the persistent solver
// ---------------------------------------------------------------------------
using SolveFn = void (*)(SolveParams);

struct Variant {
    int precision;  // AS_PREC_*
    int kmax;
    bool exact;     // clause slots == kmax (no runtime length tests)
    bool gs;        // global-storage mode (slab in global memory per trajectory, wide literals)
    int cl;         // CTAs per trajectory (thread-block cluster), global storage only
    SolveFn fn;
    size_t bytes_per_value;
    bool lean = false;  // solve_kernel_fast: FP32, plain CTDS, offset-carrying literal words
    const char* name() const { return lean ? "solve_kernel_fast" : "solve_kernel"; }
};

#define AS_VARIANT_F32(K, EX, GS, CL) \
    Variant{AS_PREC_F32_LOGA, K, EX, GS, CL, &solve_kernel<float, true, K, EX, GS, CL>, 4}
#define AS_VARIANT_F64(K, EX, GS, CL) \
    Variant{AS_PREC_F64, K, EX, GS, CL, &solve_kernel<double, false, K, EX, GS, CL>, 8}

#define AS_VARIANT_LEAN(K) \
    Variant{AS_PREC_F32_LOGA, K, true, false, 1, &solve_kernel_fast<K, false>, 4, true}
#define AS_VARIANT_LEAN_G(K) \
    Variant{AS_PREC_F32_LOGA, K, true, true, 1, &solve_kernel_fast<K, true>, 4, true}

const std::vector<Variant>& variants() {
    static const std::vector<Variant> v = {
        AS_VARIANT_LEAN(3), AS_VARIANT_LEAN(4), AS_VARIANT_LEAN_G(3), AS_VARIANT_LEAN_G(4),
        AS_VARIANT_F32(3, true, false, 1),  AS_VARIANT_F32(4, true, false, 1), AS_VARIANT_F32(2, true, false, 1),
        AS_VARIANT_F32(16, false, false, 1), AS_VARIANT_F64(3, true, false, 1), AS_VARIANT_F64(4, true, false, 1),
        AS_VARIANT_F64(16, false, false, 1), AS_VARIANT_F32(3, true, true, 1),  AS_VARIANT_F32(4, true, true, 1),
        AS_VARIANT_F32(16, false, true, 1),  AS_VARIANT_F64(3, true, true, 1),  AS_VARIANT_F64(16, false, true, 1),
        AS_VARIANT_F32(3, true, true, 4),    AS_VARIANT_F32(4, true, true, 4),  AS_VARIANT_F32(3, true, true, 8),
        AS_VARIANT_F32(4, true, true, 8),
    };
    return v;
}

size_t solver_smem(const Variant& v, const PackedProblem& q) {
    if (v.lean) {
        const FastLayout L = fast_layout(q.n, q.m, q.nslots);
        return v.gs ? (size_t)L.cs_off_g + 4 * (size_t)(q.lean_part_slots + 1) : L.bytes;
    }
    if (v.gs) return 0;
    return solve_smem_values(q.n, q.m, q.nslots) * v.bytes_per_value;
}

// Values of a trajectory's per-CTA global slab (global-storage variants).
size_t solver_slab_values(const Variant& v, const PackedProblem& q) {
    if (!v.gs) return 0;
    if (v.lean)  // the RK rows, blocked by 32 elements, clauses from the next block
        return 6 * (size_t)(row_clause_base<true>(q.n) + ((q.m + 31) & ~31));
    return solve_smem_values(q.n, q.m, q.nslots);
}

// Shared-memory variants need the compact encoding and the whole trajectory in one
// SM's shared memory; global-storage variants take any size.  The lean kernel also
// needs the plain CTDS right-hand side and its byte offsets to fit the literal words.
bool fits(const Variant& v, const PackedProblem& q, int precision, size_t smem_limit) {
    const bool kok = v.exact ? q.k == v.kmax : q.k <= v.kmax;
    if (v.precision != precision || !kok) return false;
    if (v.lean && v.gs) return standard_model(q) && q.lean_parts > 0 && solver_smem(v, q) <= smem_limit;
    if (v.lean) return standard_model(q) && q.compact && fast_layout(q.n, q.m, q.nslots).ok &&
                       solver_smem(v, q) <= smem_limit;
    if (v.gs) return true;
    return q.compact && solver_smem(v, q) <= smem_limit;
}

// Preference among fitting variants: the lean kernel, then shared memory, then exact
// K, then the smallest KMAX.
long variant_score(const Variant& v) {
    // the lean kernel with its rows in global memory still gathers and scatters in
    // shared memory: after every all-shared variant, before the general global one
    const long storage = v.gs ? (v.lean ? 50000 : 100000) : 0;
    return storage + (v.cl > 1 ? 10000 * v.cl : 0) + (v.exact ? 0 : 1000) + 2 * v.kmax + (v.lean ? 0 : 1);
}

// CTA size: the smallest clause count per thread (at least 4) that keeps the CTA at
// <= 1024 threads, then the fewest threads for that count (multiple of 32), so the
// last clause iteration is nearly full.
int preferred_bt(const PackedProblem& q) {
    int c = 4;
    while ((q.m + c - 1) / c > 1024) c++;
    const int bt = ((q.m + c - 1) / c + 31) / 32 * 32;
    return std::max(64, std::min(1024, bt));
}

// Raises a kernel's dynamic shared memory limit on the current device to at least
// `bytes`; never lowers it, so a limit that another launch group or solver (whose
// launches may sit in a captured graph) relies on stays in place.
cudaError_t raise_smem_limit(const void* fn, size_t bytes) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, fn);
    if (e != cudaSuccess) return e;
    if ((size_t)a.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// CTA size of a shared-memory launch: a trajectory of `smem_bytes` that leaves no room
// for a second CTA on its SM gets the largest CTA (more warps to hide the clause
// phase's latencies), smaller ones `bt`.
int shared_cta_threads(size_t smem_bytes, int bt, int device, int* out) {
    int per_sm = 0;
    AS_CUDA(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    *out = 2 * (smem_bytes + 2048) > (size_t)per_sm ? 1024 : bt;
    return AS_OK;
}

__global__ void stamp_deadline_kernel(unsigned long long* out, unsigned long long budget_ns) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *out = t + budget_ns;
}

}  // namespace

// ---------------------------------------------------------------------------
// handles
// ---------------------------------------------------------------------------
struct as_problem {
    HostProblem host;
    // [AS_PREC_F32_LOGA]: literals may be reordered; [AS_PREC_F64]: reference order;
    // [kLayoutPair]: the two-states-per-element RHS kernel's grouping.
    // Packed on first use of each layout.
    PackedProblem packed_[3];
    bool have_[3] = {false, false, false};
    std::mutex mu_;
    DevicePool dev[3];        // lazily uploaded for the device primitives
    DevBuf slab[3];           // per-CTA storage of the global-storage primitives
    DevBuf rhs_status;        // set by a device RHS whose bulk copy timed out (as_rhs_check)
    int rhs_status_dev = -1;  // device holding rhs_status

    int tanh = 0;       // CTDS variant (ISat implementation) and its parameters
    double q = 1.1, b = 0.0;

    const PackedProblem& packed(int layout) {
        std::lock_guard<std::mutex> lock(mu_);
        if (!have_[layout]) {
            packed_[layout] = pack(host, layout == AS_PREC_F32_LOGA ? kPackF32
                                         : layout == AS_PREC_F64    ? kPackReference
                                                                    : kPackF32Pair);
            have_[layout] = true;
        }
        packed_[layout].tanh = tanh;
        packed_[layout].q = q;
        packed_[layout].b = b;
        return packed_[layout];
    }
    bool standard_model() const { return !tanh && !(b > 0.0); }
    void pack_all() {}
};

// Device storage and the per-pass graph of the streamed solver (AS_STORAGE_STREAM).
struct StreamPlan {
    int ngroups = 0;
    std::vector<int> gprob;     // problem of each group
    std::vector<size_t> goff;   // byte offset of each group's vectors in vec
    std::vector<size_t> gcand;  // word offset of each group's candidate assignments
    DevBuf vec, lanes, tickets, active, cand;
    std::vector<std::unique_ptr<DevBuf>> vstart, vpos;  // per problem occurrence lists
    std::vector<int> have_lists, nparts;                // per problem clause parts
    cudaGraphExec_t graph = nullptr;
    long long passes = 0;       // passes of the last run
    ~StreamPlan() { if (graph) cudaGraphExecDestroy(graph); }
};

struct as_solver {
    int device = 0;
    int precision = AS_PREC_F32_LOGA;
    std::vector<PackedProblem> problems;
    std::vector<PartLayout> parts;  // per problem: clause parts of the lean global-rows form
    DevicePool pool;
    int sm_count = 0;
    size_t smem_limit = 0;

    // SatSolver defaults (SatSolver.h:60-62) and CpuRungeKutta's eps (CpuRungeKutta.cpp:43)
    double max_time = 100.0;
    int max_steps = 100000;
    int batch = 20;
    double eps = 1e-4;
    double wall_budget = 0.0;
    double last_wall = 0.0, last_cpu = 0.0;  // host wall / CPU seconds of the last as_solver_solve
    int stop_on_first = 0;
    int track_best = 0;
    int forced_bt = 0;
    int forced_cl = 0;     // CTAs per trajectory in global-storage mode (0 = automatic)
    int kernel_choice = AS_KERNEL_AUTO;  // AS_KERNEL_GENERIC: never the lean FP32 kernel
    int storage_mode = 0;  // 0 automatic, 1 shared memory, 2 global storage, 3 stream
    std::unique_ptr<StreamPlan> sp;  // streamed solver state
    int stream_parts = 0;            // clause parts per stream pass (0 = from the L2 budget)

    // trajectories
    int num_traj = 0;
    std::vector<int> traj_problem;     // user order
    std::vector<long long> traj_off;   // element offset of each trajectory (user order)
    std::vector<long long> traj_bits;  // word offset into best_bits
    long long total_values = 0;
    std::vector<int> order;            // launch order -> user trajectory
    struct Group {
        int variant, u0, u1, bt, occ, ctas;
        size_t smem, slab_off;
        long long slab_stride;
    };
    std::vector<Group> groups;

    DevBuf states, results, unit_inst, unit_state, unit_bits, queue, solved, deadline, best_bits, slab;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;  // orders a caller's stream with `stream`
    cudaGraphExec_t graph = nullptr;
    bool graph_valid = false;
    bool groups_dirty = true;
    int last_bt = 0, last_ctas = 0, last_smem = 0, last_occ = 0;
    const char* last_kernel = "";

    ~as_solver() {
        if (graph) cudaGraphExecDestroy(graph);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (stream) cudaStreamDestroy(stream);
    }
    void invalidate() { graph_valid = false; }
};

// Definitions below take C linkage from their declarations in analogsat_b200.h.

int32_t as_last_error(char* buf, int32_t buf_len) {
    if (buf && buf_len > 0) {
        std::strncpy(buf, g_last_error.c_str(), buf_len - 1);
        buf[buf_len - 1] = 0;
    }
    return (int32_t)g_last_error.size();
}

int32_t as_device_sm_count(int32_t device) {
    int dev = 0, n = 0;
    int r = current_device(device, &dev);
    if (r) return r;
    AS_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

// ---- problems ----
int32_t as_problem_create(const int32_t* literals, const int32_t* lengths, int32_t num_clauses,
                          as_problem** out) {
    if (!out || num_clauses < 0 || (num_clauses > 0 && (!literals || !lengths)))
        return fail(AS_ERR_BAD_INPUT, "as_problem_create: null argument or negative clause count");
    for (int j = 0; j < num_clauses; j++)
        if (lengths[j] < 0) return fail(AS_ERR_BAD_INPUT, "as_problem_create: negative clause length");
    auto* p = new as_problem();
    p->host.add_clauses(literals, lengths, num_clauses);
    p->pack_all();
    *out = p;
    return AS_OK;
}

int32_t as_problem_read_cnf(const char* path, as_problem** out, char* msg, int32_t msg_len) {
    if (!path || !out) return fail(AS_ERR_BAD_INPUT, "as_problem_read_cnf: null argument");
    auto* p = new as_problem();
    std::string m;
    bool ok = read_cnf(path, p->host, m);
    if (msg && msg_len > 0) {
        std::strncpy(msg, m.c_str(), msg_len - 1);
        msg[msg_len - 1] = 0;
    }
    if (!ok) {
        delete p;
        return fail(AS_ERR_IO, "as_problem_read_cnf: " + m);
    }
    p->pack_all();
    *out = p;
    return AS_OK;
}

int32_t as_problem_read_cnf_device(const char* path, int32_t device, as_problem** out, char* msg,
                                   int32_t msg_len) {
    if (!path || !out) return fail(AS_ERR_BAD_INPUT, "as_problem_read_cnf_device: null argument");
    auto put = [&](const std::string& m) {
        if (msg && msg_len > 0) {
            std::strncpy(msg, m.c_str(), msg_len - 1);
            msg[msg_len - 1] = 0;
        }
    };
    FILE* f = std::fopen(path, "r");
    if (!f) {
        put("file open failed");
        return fail(AS_ERR_IO, "as_problem_read_cnf_device: file open failed");
    }
    std::unique_ptr<FILE, int (*)(FILE*)> fg(f, std::fclose);
    int n = -1, m = -1;
    std::string mm;
    if (!read_cnf_header(f, n, m, mm)) {
        put(mm);
        return fail(AS_ERR_IO, "as_problem_read_cnf_device: " + mm);
    }
    std::unique_ptr<as_problem> p(new as_problem());
    if (n == 0 || m == 0) {
        put("empty problem");
        *out = p.release();
        return AS_OK;
    }
    const long start = std::ftell(f);
    if (start < 0 || std::fseek(f, 0, SEEK_END) != 0) return fail(AS_ERR_IO, "as_problem_read_cnf_device: seek failed");
    const long end = std::ftell(f);
    if (end < start || std::fseek(f, start, SEEK_SET) != 0)
        return fail(AS_ERR_IO, "as_problem_read_cnf_device: seek failed");
    const size_t len = (size_t)(end - start);
    int prev = 0;
    AS_CUDA(cudaGetDevice(&prev));
    AS_CUDA(cudaSetDevice(device));
    struct Restore {
        int d;
        ~Restore() { cudaSetDevice(d); }
    } restore{prev};
    std::vector<int32_t> lits, lens;
    cudaError_t ce = cudaSuccess;
    const bool ok = asb::parse_cnf_body(f, len, m, lits, lens, mm, ce);
    if (ce != cudaSuccess) return fail(AS_ERR_CUDA, "as_problem_read_cnf_device: " + mm);
    put(mm);
    if (!ok) return fail(AS_ERR_IO, "as_problem_read_cnf_device: " + mm);
    p->host.set_clauses(std::move(lits), lens);
    *out = p.release();
    return AS_OK;
}

int32_t as_problem_write_cnf(const as_problem* p, const char* path) {
    if (!p || !path) return fail(AS_ERR_BAD_INPUT, "as_problem_write_cnf: null argument");
    return write_cnf(path, p->host) ? AS_OK : fail(AS_ERR_IO, "as_problem_write_cnf: file open failed");
}

int32_t as_problem_get_nmk(const as_problem* p, int32_t* n, int32_t* m, int32_t* k) {
    if (!p) return fail(AS_ERR_BAD_INPUT, "as_problem_get_nmk: null problem");
    if (n) *n = p->host.n;
    if (m) *m = p->host.m;
    if (k) *k = p->host.k;
    return AS_OK;
}

int32_t as_problem_num_literals(const as_problem* p) {
    if (!p) return fail(AS_ERR_BAD_INPUT, "as_problem_num_literals: null problem");
    return (int32_t)p->host.storage.size();
}

int32_t as_problem_get_clauses(const as_problem* p, int32_t* literals, int32_t* lengths) {
    if (!p || !literals || !lengths) return fail(AS_ERR_BAD_INPUT, "as_problem_get_clauses: null argument");
    size_t o = 0;
    for (int j = 0; j < p->host.m; j++) {
        lengths[j] = p->host.length[j];
        for (int i = 0; i < p->host.length[j]; i++) literals[o++] = p->host.storage[p->host.start[j] + i];
    }
    return AS_OK;
}

int32_t as_problem_layout_stats(const as_problem* p, int32_t precision, int32_t* nslots,
                                int32_t* max_degree, int64_t* bank_wavefronts, int32_t* compact) {
    if (!p || (precision != AS_PREC_F32_LOGA && precision != AS_PREC_F64 && precision != AS_LAYOUT_F32_PAIR))
        return fail(AS_ERR_BAD_INPUT, "as_problem_layout_stats: bad argument");
    const auto& q = const_cast<as_problem*>(p)->packed(precision);
    if (nslots) *nslots = q.nslots;
    if (max_degree) *max_degree = q.max_degree;
    if (bank_wavefronts) *bank_wavefronts = q.bank_wavefronts;
    if (compact) *compact = q.compact ? 1 : 0;
    return AS_OK;
}

void as_problem_free(as_problem* p) { delete p; }

int32_t as_problem_set_model(as_problem* p, int32_t model, double q) {
    if (!p || (model != AS_MODEL_CTDS && model != AS_MODEL_TANH) || !std::isfinite(q))
        return fail(AS_ERR_BAD_INPUT, "as_problem_set_model: bad argument");
    std::lock_guard<std::mutex> lock(p->mu_);
    p->tanh = model == AS_MODEL_TANH ? 1 : 0;
    p->q = q;
    for (auto& d : p->dev) d.device = -1;  // re-upload the instance record
    return AS_OK;
}

int32_t as_problem_set_bias(as_problem* p, double b) {
    if (!p || !(b >= 0.0) || !std::isfinite(b)) return fail(AS_ERR_BAD_INPUT, "as_problem_set_bias: need b >= 0");
    std::lock_guard<std::mutex> lock(p->mu_);
    p->b = b;
    for (auto& d : p->dev) d.device = -1;
    return AS_OK;
}

int32_t as_problem_get_model(const as_problem* p, int32_t* model, double* q, double* b) {
    if (!p) return fail(AS_ERR_BAD_INPUT, "null problem");
    if (model) *model = p->tanh ? AS_MODEL_TANH : AS_MODEL_CTDS;
    if (q) *q = p->q;
    if (b) *b = p->b;
    return AS_OK;
}

// ---- device primitives ----
namespace {

int ensure_uploaded(as_problem* p, int prec) {
    if (p->host.m == 0 || p->host.k == 0) return fail(AS_ERR_NO_PROBLEM, "SAT problem has not been set");
    int dev = 0;
    AS_CUDA(cudaGetDevice(&dev));
    if (p->dev[prec].device == dev) return AS_OK;
    std::vector<const PackedProblem*> v{&p->packed(prec)};
    return p->dev[prec].upload(v, dev);
}

// Grid-stride launch of a per-state kernel: the shared-memory form when the state
// fits one SM, else the global-storage form with a per-CTA slab owned by the problem
// handle (grown on demand; calls on one handle must not overlap).
template <typename T, typename OUT>
int launch_per_state(as_problem* p, int prec, void (*fs)(DevInstance, const T*, OUT*, int, long long, T*, long long),
                     void (*fg)(DevInstance, const T*, OUT*, int, long long, T*, long long), int bt,
                     size_t vals, bool compact, const T* x, OUT* out, int ns, long long stride,
                     cudaStream_t st) {
    int dev = 0, sms = 0, optin = 0, occ = 0;
    AS_CUDA(cudaGetDevice(&dev));
    AS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    AS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t smem = vals * sizeof(T);
    if (compact && smem + 1024 <= (size_t)optin) {
        AS_CUDA(raise_smem_limit((const void*)fs, smem));
        AS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fs, bt, smem));
        const int grid = std::max(1, std::min(ns, sms * std::max(occ, 1)));
        fs<<<grid, bt, smem, st>>>(p->dev[prec].host_inst[0], x, out, ns, stride, (T*)nullptr, 0ll);
    } else {
        AS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fg, bt, 0));
        const int grid = std::max(1, std::min(ns, sms * std::max(occ, 1)));
        const long long slab_stride = (long long)((vals + 63) / 64 * 64);
        AS_CUDA(p->slab[prec].alloc((size_t)grid * slab_stride * sizeof(T)));
        fg<<<grid, bt, 0, st>>>(p->dev[prec].host_inst[0], x, out, ns, stride, p->slab[prec].as<T>(),
                                 slab_stride);
    }
    AS_CUDA(cudaGetLastError());
    return AS_OK;
}

// Two states per CTA pass with packed FP32x2 arithmetic (FP32, compact instances whose
// pair-kernel footprint fits one SM's shared memory); *done = false leaves the call to
// the one-state kernel.
template <bool LOGA, int KMAX, bool EXACT>
int launch_rhs_pair(as_problem* p, const float* x, float* d, int ns, cudaStream_t st, bool* done) {
    constexpr int BT = 1024;
    *done = false;
    if ((reinterpret_cast<uintptr_t>(x) & 3u) || !p->standard_model()) return AS_OK;
    const auto& q = p->packed(kLayoutPair);
    int dev = 0, sms = 0, optin = 0, occ = 0;
    AS_CUDA(cudaGetDevice(&dev));
    AS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    AS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t smem = rhs2_smem_bytes(q.n, q.m, q.nslots);
    constexpr int CPT = 5, VPT = 1;  // instances whose footprint fits have M <= 5 * 1024
    if (!q.compact || smem + 1024 > (size_t)optin || q.m > CPT * BT || q.n > VPT * BT) return AS_OK;
    int r = ensure_uploaded(p, kLayoutPair);
    if (r) return r;
    auto fn = &rhs_pair_kernel<LOGA, KMAX, EXACT, BT, CPT, VPT>;
    AS_CUDA(raise_smem_limit((const void*)fn, smem));
    AS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, BT, smem));
    if (occ < 1) return AS_OK;
    const int grid = std::max(1, std::min((ns + 1) / 2, sms * occ));
    // bulk stores need dxdt congruent with x mod 16 bytes (same staging offsets)
    const int bulk_out = ((reinterpret_cast<uintptr_t>(x) - reinterpret_cast<uintptr_t>(d)) & 15u) == 0;
    if (p->rhs_status_dev != dev) {
        AS_CUDA(p->rhs_status.alloc(sizeof(int)));
        AS_CUDA(cudaMemset(p->rhs_status.p, 0, sizeof(int)));
        p->rhs_status_dev = dev;
    }
    fn<<<grid, BT, smem, st>>>(p->dev[kLayoutPair].host_inst[0], x, d, ns, (long long)(q.n + q.m),
                               bulk_out, p->rhs_status.as<int>());
    AS_CUDA(cudaGetLastError());
    *done = true;
    return AS_OK;
}

template <typename T, bool LOGA, int KMAX, bool EXACT>
int launch_rhs(as_problem* p, const T* x, T* d, int ns, cudaStream_t st) {
    constexpr int BT = 512;
    constexpr int prec = sizeof(T) == 8 ? AS_PREC_F64 : AS_PREC_F32_LOGA;
    if constexpr (sizeof(T) == 4 && EXACT) {
        bool done = false;
        const int r = launch_rhs_pair<LOGA, KMAX, EXACT>(p, x, d, ns, st, &done);
        if (r || done) return r;
    }
    const auto& q = p->packed(prec);
    return launch_per_state<T, T>(p, prec, &rhs_batch_kernel<T, LOGA, KMAX, EXACT, BT, false>,
                                  &rhs_batch_kernel<T, LOGA, KMAX, EXACT, BT, true>, BT,
                                  rhs_smem_values(q.n, q.m, q.nslots), q.compact, x, d, ns,
                                  (long long)(q.n + q.m), st);
}

template <typename T, bool LOGA>
int dispatch_rhs(as_problem* p, const T* x, T* d, int ns, void* stream) {
    if (!p || !x || !d || ns < 0) return fail(AS_ERR_BAD_INPUT, "as_rhs: null argument");
    if (ns == 0) return AS_OK;
    constexpr int prec = sizeof(T) == 8 ? AS_PREC_F64 : AS_PREC_F32_LOGA;
    int r = ensure_uploaded(p, prec);
    if (r) return r;
    cudaStream_t st = (cudaStream_t)stream;
    const int k = p->packed(prec).k;
    if (k == 3) return launch_rhs<T, LOGA, 3, true>(p, x, d, ns, st);
    if (k == 4) return launch_rhs<T, LOGA, 4, true>(p, x, d, ns, st);
    if (k <= 16) return launch_rhs<T, LOGA, 16, false>(p, x, d, ns, st);
    return fail(AS_ERR_UNSUPPORTED, "clause length > 16 is not supported");
}

template <typename T, int KMAX, bool EXACT>
int launch_viol(as_problem* p, const T* x, int* c, int ns, cudaStream_t st) {
    constexpr int BT = 256;
    constexpr int prec = sizeof(T) == 8 ? AS_PREC_F64 : AS_PREC_F32_LOGA;
    const auto& q = p->packed(prec);
    return launch_per_state<T, int>(p, prec, &viol_batch_kernel<T, KMAX, EXACT, BT, false>,
                                    &viol_batch_kernel<T, KMAX, EXACT, BT, true>, BT,
                                    (size_t)((q.n + 1 + 3) & ~3), q.compact, x, c, ns,
                                    (long long)(q.n + q.m), st);
}

template <typename T>
int dispatch_viol(as_problem* p, const T* x, int* c, int ns, void* stream) {
    if (!p || !x || !c || ns < 0) return fail(AS_ERR_BAD_INPUT, "as_violations: null argument");
    if (ns == 0) return AS_OK;
    constexpr int prec = sizeof(T) == 8 ? AS_PREC_F64 : AS_PREC_F32_LOGA;
    int r = ensure_uploaded(p, prec);
    if (r) return r;
    cudaStream_t st = (cudaStream_t)stream;
    const int k = p->packed(prec).k;
    if (k == 3) return launch_viol<T, 3, true>(p, x, c, ns, st);
    if (k == 4) return launch_viol<T, 4, true>(p, x, c, ns, st);
    if (k <= 16) return launch_viol<T, 16, false>(p, x, c, ns, st);
    return fail(AS_ERR_UNSUPPORTED, "clause length > 16 is not supported");
}

}  // namespace

int32_t as_rhs_f32(as_problem* p, const float* x, float* dxdt, int32_t num_states, int32_t logspace,
                   void* stream) {
    return logspace ? dispatch_rhs<float, true>(p, x, dxdt, num_states, stream)
                    : dispatch_rhs<float, false>(p, x, dxdt, num_states, stream);
}

int32_t as_rhs_check(as_problem* p, void* stream) {
    if (!p) return fail(AS_ERR_BAD_INPUT, "as_rhs_check: null problem");
    AS_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (p->rhs_status_dev < 0) return AS_OK;  // no bulk-copy RHS has run
    int dev = 0, word = 0;
    AS_CUDA(cudaGetDevice(&dev));
    if (dev != p->rhs_status_dev) AS_CUDA(cudaSetDevice(p->rhs_status_dev));
    cudaError_t e = cudaMemcpy(&word, p->rhs_status.p, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && word) e = cudaMemset(p->rhs_status.p, 0, sizeof(int));
    if (dev != p->rhs_status_dev) cudaSetDevice(dev);
    if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("as_rhs_check: ") + cudaGetErrorString(e));
    if (word)
        return fail(AS_ERR_TIMEOUT, "as_rhs_f32: a bulk copy did not complete within 2 s; the states "
                                    "of the affected CTA hold NaN");
    return AS_OK;
}

int32_t as_rhs_f64(as_problem* p, const double* x, double* dxdt, int32_t num_states, void* stream) {
    return dispatch_rhs<double, false>(p, x, dxdt, num_states, stream);
}

int32_t as_violations_f32(as_problem* p, const float* x, int32_t* counts, int32_t num_states,
                          void* stream) {
    return dispatch_viol<float>(p, x, counts, num_states, stream);
}

int32_t as_violations_f64(as_problem* p, const double* x, int32_t* counts, int32_t num_states,
                          void* stream) {
    return dispatch_viol<double>(p, x, counts, num_states, stream);
}

// ---- solver ----
int32_t as_solver_create(const as_problem* const* problems, int32_t num_problems, int32_t precision,
                         int32_t device, as_solver** out) {
    if (!out || !problems || num_problems <= 0)
        return fail(AS_ERR_BAD_INPUT, "as_solver_create: need at least one problem");
    if (precision != AS_PREC_F32_LOGA && precision != AS_PREC_F64)
        return fail(AS_ERR_BAD_INPUT, "as_solver_create: unknown precision");
    for (int i = 0; i < num_problems; i++) {
        if (!problems[i]) return fail(AS_ERR_BAD_INPUT, "as_solver_create: null problem");
        if (problems[i]->host.k == 0) return fail(AS_ERR_NO_PROBLEM, "SAT problem has not been set");
    }
    std::unique_ptr<as_solver> s(new as_solver());
    int r = current_device(device, &s->device);
    if (r) return r;
    s->precision = precision;
    for (int i = 0; i < num_problems; i++) s->problems.push_back(const_cast<as_problem*>(problems[i])->packed(precision));
    int optin = 0;
    AS_CUDA(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device));
    AS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device));
    s->smem_limit = (size_t)optin - 1024;  // static shared memory of the kernel
    // FP32 plain-CTDS instances beyond the all-shared lean layout: clause parts for the
    // lean kernel's global-rows form, the fewest parts whose slots fit one SM
    s->parts.assign(num_problems, PartLayout());
    if (precision == AS_PREC_F32_LOGA)
        for (int i = 0; i < num_problems; i++) {
            auto& q = s->problems[i];
            if (!standard_model(q) || (q.k != 3 && q.k != 4) || q.n >= 8191) continue;
            const FastLayout L = fast_layout(q.n, q.m, q.nslots);
            if (q.compact && L.ok && L.bytes <= s->smem_limit) continue;  // the all-shared form takes it
            const HostProblem& hp = problems[i]->host;
            for (int np = 1; np <= 4; np++) {
                PartLayout PL;
                if (!pack_parts(hp, q, np, PL)) break;
                if ((size_t)L.cs_off_g + 4 * (size_t)(PL.max_slots + 1) <= s->smem_limit) {
                    q.lean_parts = np;
                    q.lean_part_slots = PL.max_slots;
                    s->parts[i] = std::move(PL);
                    break;
                }
            }
        }
    std::vector<const PackedProblem*> pk;
    for (auto& q : s->problems) pk.push_back(&q);
    r = s->pool.upload(pk, s->device, &s->parts);
    if (r) return r;
    AS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    for (auto& q : s->problems) {
        bool any = false;
        for (auto& v : variants()) any = any || fits(v, q, precision, s->smem_limit);
        if (!any)
            return fail(AS_ERR_UNSUPPORTED,
                        "instance N=" + std::to_string(q.n) + " M=" + std::to_string(q.m) +
                            " K=" + std::to_string(q.k) + " exceeds every compiled launch shape");
    }
    AS_CUDA(s->queue.alloc(64 * sizeof(int)));
    AS_CUDA(s->solved.alloc(sizeof(int) * s->problems.size()));
    AS_CUDA(s->deadline.alloc(sizeof(unsigned long long)));
    *out = s.release();
    return AS_OK;
}

void as_solver_free(as_solver* s) { delete s; }

int32_t as_solver_set_max_time(as_solver* s, double v) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (!(v > 0.0)) return fail(AS_ERR_BAD_INPUT, "Max time must be positive");
    s->max_time = v; s->invalidate();
    return AS_OK;
}
int32_t as_solver_set_max_steps(as_solver* s, int32_t v) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (v < 1) return fail(AS_ERR_BAD_INPUT, "Max iterations must be positive");
    s->max_steps = v; s->invalidate();
    return AS_OK;
}
int32_t as_solver_set_batch_size(as_solver* s, int32_t v) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (v < 1) return fail(AS_ERR_BAD_INPUT, "Batch size must be positive");
    s->batch = v; s->invalidate();
    return AS_OK;
}
int32_t as_solver_set_epsilon(as_solver* s, double v) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (!(v >= 1e-16 && v <= 1.0)) return fail(AS_ERR_BAD_INPUT, "epsilon must be between 1e-16 and 1");
    s->eps = v; s->invalidate();
    return AS_OK;
}
int32_t as_solver_set_wall_budget(as_solver* s, double v) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (!(v >= 0.0)) return fail(AS_ERR_BAD_INPUT, "wall budget must be >= 0");
    s->wall_budget = v; s->invalidate();
    return AS_OK;
}
int32_t as_solver_set_stop_on_first(as_solver* s, int32_t f) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    s->stop_on_first = f ? 1 : 0; s->invalidate();
    return AS_OK;
}
int32_t as_solver_set_track_best(as_solver* s, int32_t f) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    s->track_best = f ? 1 : 0; s->invalidate();
    return AS_OK;
}

namespace {

// Record the trajectories' problems and state offsets (user order) and size the
// state buffer.  Grouping by launch shape happens lazily in build_groups.
int plan_units(as_solver* s, const int32_t* problem_index, int num_traj) {
    if (num_traj <= 0 || !problem_index) return fail(AS_ERR_BAD_INPUT, "need at least one trajectory");
    const int np = (int)s->problems.size();
    for (int t = 0; t < num_traj; t++)
        if (problem_index[t] < 0 || problem_index[t] >= np)
            return fail(AS_ERR_BAD_INPUT, "problem index out of range");
    // the same trajectories as the last call: buffers, unit tables and the captured
    // solve stay valid, only the state values change
    if (num_traj == s->num_traj && s->states.p &&
        std::equal(problem_index, problem_index + num_traj, s->traj_problem.begin()))
        return AS_OK;
    s->num_traj = num_traj;
    s->traj_problem.assign(problem_index, problem_index + num_traj);
    s->traj_off.resize(num_traj);
    s->traj_bits.resize(num_traj);
    long long off = 0, bo = 0;
    for (int t = 0; t < num_traj; t++) {
        const auto& q = s->problems[problem_index[t]];
        s->traj_off[t] = off;
        off += q.n + q.m;
        s->traj_bits[t] = bo;
        bo += (q.n + 31) / 32;
    }
    s->total_values = off;
    const size_t vb = s->precision == AS_PREC_F64 ? 8 : 4;
    AS_CUDA(s->states.alloc((size_t)off * vb));
    AS_CUDA(s->results.alloc(sizeof(UnitResult) * num_traj));
    AS_CUDA(s->unit_inst.alloc(sizeof(int) * num_traj));
    AS_CUDA(s->unit_state.alloc(sizeof(long long) * num_traj));
    AS_CUDA(s->unit_bits.alloc(sizeof(long long) * num_traj));
    AS_CUDA(s->best_bits.alloc(sizeof(uint32_t) * std::max<long long>(bo, 1)));
    s->groups_dirty = true;
    s->invalidate();
    return AS_OK;
}

// Pick the launch shape of every problem (smallest CTA that holds it, or the forced
// shape), order the trajectories by (shape, problem) and upload the unit tables.
int build_groups(as_solver* s) {
    const auto& vs = variants();
    const int np = (int)s->problems.size();
    const int num_traj = s->num_traj;
    std::vector<int> pv(np, -1);
    for (int p = 0; p < np; p++) {
        const auto& q = s->problems[p];
        long best = -1;
        for (int i = 0; i < (int)vs.size(); i++) {
            const auto& v = vs[i];
            if (!fits(v, q, s->precision, s->smem_limit)) continue;
            if ((s->storage_mode == 1 && v.gs) || (s->storage_mode == 2 && !v.gs)) continue;
            if (v.lean && s->kernel_choice == AS_KERNEL_GENERIC) continue;
            const long score = variant_score(v);
            if (pv[p] < 0 || score < best) { best = score; pv[p] = i; }
        }
        if (pv[p] < 0)
            return fail(AS_ERR_UNSUPPORTED, "no compiled launch shape fits problem " + std::to_string(p));
    }
    // global-storage problems with few trajectories: spread each trajectory over a
    // cluster of CTAs so that all trajectories run at once on the whole GPU
    {
        std::vector<int> per_problem(np, 0);
        for (int t = 0; t < num_traj; t++) per_problem[s->traj_problem[t]]++;
        long gs_units = 0;
        for (int p = 0; p < np; p++)
            if (vs[pv[p]].gs) gs_units += per_problem[p];
        bool bias = false;  // the bias term's clause-weight sum is reduced per CTA
        for (const auto& q : s->problems) bias |= q.b > 0.0 || q.tanh;
        int want_cl = 1;
        if (s->forced_cl) want_cl = s->forced_cl;
        else if (!bias)
            while (want_cl < 8 && gs_units > 0 && gs_units * want_cl * 2 <= s->sm_count) want_cl *= 2;
        if (bias && want_cl > 1)
            return fail(AS_ERR_UNSUPPORTED, "clusters of CTAs per trajectory do not support the bias term "
                                            "or the tanh variant");
        if (want_cl > 1 && !s->forced_bt) {
            for (int p = 0; p < np; p++) {
                const Variant& cur = vs[pv[p]];
                if (!cur.gs) continue;
                for (int i = 0; i < (int)vs.size(); i++)
                    if (vs[i].gs && vs[i].cl == want_cl && vs[i].precision == cur.precision &&
                        vs[i].kmax == cur.kmax && vs[i].exact == cur.exact)
                        pv[p] = i;
            }
        }
    }
    const auto& pi = s->traj_problem;
    // Within a launch shape the work queue deals the problems round-robin (the r-th
    // trajectory of every problem before the (r+1)-th of any), so the trajectories
    // running at once belong to different problems: with stop-on-first an instance's
    // restarts then run a few at a time instead of filling the GPU together and being
    // stopped together.
    std::vector<int> rank(num_traj), seen(np, 0);
    for (int t = 0; t < num_traj; t++) rank[t] = seen[pi[t]]++;
    s->order.resize(num_traj);
    for (int t = 0; t < num_traj; t++) s->order[t] = t;
    std::stable_sort(s->order.begin(), s->order.end(), [&](int a, int b) {
        const int va = pv[pi[a]], vb = pv[pi[b]];
        if (va != vb) return va < vb;
        if (rank[a] != rank[b]) return rank[a] < rank[b];
        return pi[a] < pi[b];
    });
    s->groups.clear();
    size_t slab_total = 0;
    for (int u = 0; u < num_traj;) {
        const int vi = pv[pi[s->order[u]]];
        const Variant& v = vs[vi];
        int e = u, bt = 64;
        size_t vals = 0, sbytes = 0;
        while (e < num_traj && pv[pi[s->order[e]]] == vi) {
            const auto& q = s->problems[pi[s->order[e]]];
            bt = std::max(bt, preferred_bt(q));
            vals = std::max(vals, solver_slab_values(v, q));
            sbytes = std::max(sbytes, solver_smem(v, q));
            e++;
        }
        as_solver::Group G;
        G.variant = vi;
        G.u0 = u;
        G.u1 = e;
        // global storage: 512 threads (two CTAs per SM) while the in-flight slabs fit in
        // L2, else 1,024 (one per SM, half the slabs)
        int gs_bt = 512;
        if (v.gs && v.cl == 1 && !v.lean) {
            int l2 = 0;
            AS_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, s->device));
            if (2.0 * s->sm_count * (double)vals * v.bytes_per_value > 0.75 * l2) gs_bt = 1024;
        }
        // shared memory: a trajectory that leaves no room for a second CTA on the SM gets
        // the largest CTA (more warps to hide the clause phase's latencies)
        int sm_bt = bt;
        if (!v.gs || v.lean) {
            const int r = shared_cta_threads(sbytes, bt, s->device, &sm_bt);
            if (r) return r;
        }
        G.bt = s->forced_bt ? s->forced_bt : (v.gs && !v.lean ? (v.cl > 1 ? 1024 : gs_bt) : sm_bt);
        G.smem = sbytes;
        AS_CUDA(raise_smem_limit((const void*)v.fn, G.smem));
        int occ = 0;
        if (v.cl > 1) {
            AS_CUDA(cudaFuncSetAttribute(v.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr;
            attr.id = cudaLaunchAttributeClusterDimension;
            attr.val.clusterDim.x = v.cl;
            attr.val.clusterDim.y = 1;
            attr.val.clusterDim.z = 1;
            cfg.gridDim = dim3(v.cl * std::max(1, e - u));
            cfg.blockDim = dim3(G.bt);
            cfg.dynamicSmemBytes = G.smem;
            cfg.attrs = &attr;
            cfg.numAttrs = 1;
            AS_CUDA(cudaOccupancyMaxActiveClusters(&occ, (const void*)v.fn, &cfg));
            if (occ < 1) return fail(AS_ERR_UNSUPPORTED, "cluster launch shape does not fit");
            G.occ = occ;
            G.ctas = std::min(e - u, occ) * v.cl;  // clusters resident at once x CTAs per cluster
        } else {
            AS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v.fn, G.bt, G.smem));
            if (occ < 1) return fail(AS_ERR_UNSUPPORTED, "launch shape does not fit on an SM");
            G.occ = occ;
            G.ctas = std::min(e - u, s->sm_count * occ);
        }
        G.slab_stride = v.gs ? (long long)((vals + 63) / 64 * 64) : 0;
        G.slab_off = slab_total;
        slab_total += (size_t)(G.ctas / v.cl) * (size_t)G.slab_stride * v.bytes_per_value;
        s->groups.push_back(G);
        u = e;
    }
    if (slab_total) AS_CUDA(s->slab.alloc(slab_total));
    std::vector<int> ui(num_traj);
    std::vector<long long> us(num_traj), ub(num_traj);
    for (int u = 0; u < num_traj; u++) {
        ui[u] = pi[s->order[u]];
        us[u] = s->traj_off[s->order[u]];
        ub[u] = s->traj_bits[s->order[u]];
    }
    if (s->groups.size() + 1 > s->queue.bytes / sizeof(int))
        AS_CUDA(s->queue.alloc(sizeof(int) * (s->groups.size() + 1)));
    AS_CUDA(cudaMemcpy(s->unit_inst.p, ui.data(), sizeof(int) * num_traj, cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemcpy(s->unit_state.p, us.data(), sizeof(long long) * num_traj, cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemcpy(s->unit_bits.p, ub.data(), sizeof(long long) * num_traj, cudaMemcpyHostToDevice));
    s->groups_dirty = false;
    s->invalidate();
    return AS_OK;
}

template <typename SRC>
int set_states_host(as_solver* s, const int32_t* pi, int nt, const SRC* src) {
    if (!s || !src) return fail(AS_ERR_BAD_INPUT, "as_solver_set_states: null argument");
    AS_CUDA(cudaSetDevice(s->device));
    int r = plan_units(s, pi, nt);
    if (r) return r;
    const size_t n = (size_t)s->total_values;
    if (s->precision == AS_PREC_F64) {
        if (sizeof(SRC) == 8) {
            AS_CUDA(cudaMemcpyAsync(s->states.p, src, n * 8, cudaMemcpyHostToDevice, s->stream));
        } else {
            std::vector<double> tmp(src, src + n);
            AS_CUDA(cudaMemcpyAsync(s->states.p, tmp.data(), n * 8, cudaMemcpyHostToDevice, s->stream));
            AS_CUDA(cudaStreamSynchronize(s->stream));
        }
    } else {
        if (sizeof(SRC) == 4) {
            AS_CUDA(cudaMemcpyAsync(s->states.p, src, n * 4, cudaMemcpyHostToDevice, s->stream));
        } else {
            std::vector<float> tmp(src, src + n);
            AS_CUDA(cudaMemcpyAsync(s->states.p, tmp.data(), n * 4, cudaMemcpyHostToDevice, s->stream));
            AS_CUDA(cudaStreamSynchronize(s->stream));
        }
    }
    return AS_OK;
}

int record_solve(as_solver* s, cudaStream_t st) {
    const auto& vs = variants();
    AS_CUDA(cudaMemsetAsync(s->queue.p, 0, s->queue.bytes, st));
    AS_CUDA(cudaMemsetAsync(s->solved.p, 0, s->solved.bytes, st));
    const bool have_deadline = s->wall_budget > 0.0;
    if (have_deadline) {
        stamp_deadline_kernel<<<1, 1, 0, st>>>(s->deadline.as<unsigned long long>(),
                                               (unsigned long long)(s->wall_budget * 1e9));
        AS_CUDA(cudaGetLastError());
    }
    for (size_t g = 0; g < s->groups.size(); g++) {
        const auto& G = s->groups[g];
        const Variant& v = vs[G.variant];
        const size_t smem = G.smem;
        const int occ = G.occ, ctas = G.ctas, units = G.u1 - G.u0;
        SolveParams P;
        P.inst = s->pool.inst.as<DevInstance>();
        P.unit_inst = s->unit_inst.as<int>() + G.u0;
        P.unit_state = s->unit_state.as<long long>() + G.u0;
        P.states = s->states.p;
        P.results = s->results.as<UnitResult>() + G.u0;
        P.queue_head = s->queue.as<int>() + g;
        P.inst_solved = s->solved.as<int>();
        P.best_bits = s->track_best ? s->best_bits.as<uint32_t>() : nullptr;
        P.unit_bits = s->unit_bits.as<long long>() + G.u0;
        P.num_units = units;
        P.maxsteps = s->max_steps;
        P.batch = s->batch;
        P.stop_on_first = s->stop_on_first;
        P.eps = s->eps;
        P.tmax = s->max_time;
        P.deadline = have_deadline ? s->deadline.as<unsigned long long>() : nullptr;
        P.slab = v.gs ? static_cast<char*>(s->slab.p) + G.slab_off : nullptr;
        P.slab_stride = G.slab_stride;
        void* args[] = {&P};
        if (v.cl > 1) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr;
            attr.id = cudaLaunchAttributeClusterDimension;
            attr.val.clusterDim.x = v.cl;
            attr.val.clusterDim.y = 1;
            attr.val.clusterDim.z = 1;
            cfg.gridDim = dim3(ctas);
            cfg.blockDim = dim3(G.bt);
            cfg.dynamicSmemBytes = smem;
            cfg.stream = st;
            cfg.attrs = &attr;
            cfg.numAttrs = 1;
            AS_CUDA(cudaLaunchKernelExC(&cfg, (const void*)v.fn, args));
        } else {
            AS_CUDA(cudaLaunchKernel((const void*)v.fn, dim3(ctas), dim3(G.bt), args, smem, st));
        }
        s->last_bt = G.bt; s->last_ctas = ctas; s->last_smem = (int)smem; s->last_occ = occ;
        s->last_kernel = v.name();
    }
    return AS_OK;
}

// ---------------------------------------------------------------------------
// Streamed solver (AS_STORAGE_STREAM, as_stream.cuh): host side
// ---------------------------------------------------------------------------
constexpr long long kStreamAutoElements = 1ll << 19;  // AS_STORAGE_AUTO: N + M from here on

bool use_stream(const as_solver* s) {
    if (s->storage_mode == 3) return true;
    if (s->storage_mode != 0 || s->num_traj <= 0) return false;
    for (const auto& q : s->problems)
        if (!standard_model(q)) return false;  // the streamed kernels have the CpuSat RHS only
    for (int t = 0; t < s->num_traj; t++) {
        const auto& q = s->problems[s->traj_problem[t]];
        if ((long long)q.n + q.m < kStreamAutoElements) return false;
    }
    return true;
}

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

size_t stream_group_bytes(const PackedProblem& q, size_t vbytes) {
    const long long E = (long long)q.n + q.m;
    return 6 * round256((size_t)E * kLanes * vbytes) + round256((size_t)(q.n + 1) * kLanes * vbytes) +
           round256((size_t)q.k * q.mp * kLanes * vbytes) + round256((size_t)q.n * kLanes * vbytes);
}

template <typename T>
StreamArgs<T> stream_args(as_solver* s, int g, const unsigned long long* deadline) {
    StreamPlan& P = *s->sp;
    const int p = P.gprob[g];
    const auto& q = s->problems[p];
    const size_t vb = round256((size_t)((long long)q.n + q.m) * kLanes * sizeof(T));
    char* base = static_cast<char*>(P.vec.p) + P.goff[g];
    StreamArgs<T> A;
    A.I = s->pool.host_inst[p];
    A.X = reinterpret_cast<T*>(base);
    A.K1 = reinterpret_cast<T*>(base + vb);
    A.K2 = reinterpret_cast<T*>(base + 2 * vb);
    A.K3 = reinterpret_cast<T*>(base + 3 * vb);
    A.K4 = reinterpret_cast<T*>(base + 4 * vb);
    A.K5 = reinterpret_cast<T*>(base + 5 * vb);
    A.SY = reinterpret_cast<T*>(base + 6 * vb);
    A.CS = reinterpret_cast<T*>(base + 6 * vb + round256((size_t)(q.n + 1) * kLanes * sizeof(T)));
    A.lanes = P.lanes.as<LaneState>() + (size_t)g * kLanes;
    A.vstart = P.vstart[p]->as<int>();
    A.vpos = P.vpos[p]->as<int>();
    A.ACC = reinterpret_cast<T*>(base + 6 * vb + round256((size_t)(q.n + 1) * kLanes * sizeof(T)) +
                                 round256((size_t)q.k * q.mp * kLanes * sizeof(T)));
    A.m0 = 0;
    A.m1 = q.m;
    A.part = 0;
    A.nparts = P.nparts[p];
    A.tickets = P.tickets.as<int>() + 2 * g;
    A.active = P.active.as<int>() + g;
    A.cand_bits = P.cand.as<uint32_t>() + P.gcand[g];
    A.best_bits = s->track_best ? s->best_bits.as<uint32_t>() : nullptr;
    A.unit_bits = s->unit_bits.as<long long>();
    A.inst_solved = s->solved.as<int>();
    A.deadline = deadline;
    A.pidx = p;
    A.S = 1;
    A.batch = s->batch;
    A.maxsteps = s->max_steps;
    A.stop_on_first = s->stop_on_first;
    A.eps = s->eps;
    A.tmax = s->max_time;
    return A;
}


// Occurrence lists of a packed problem's internal variables: the contribution rows
// q * mp + m of its literals, in the order of its SELL row (public clause order), and
// their split into clause parts.  Parts are ranges of public clause index; they need
// internal clause order = public order (the wide packing keeps it), else one part.
// vstart holds nparts + 1 arrays of n offsets: part p of variable v is
// [vstart[p n + v], vstart[(p + 1) n + v]).
int stream_lists(as_solver* s, int p) {
    StreamPlan& P = *s->sp;
    const auto& q = s->problems[p];
    bool identity = true;
    for (int m = 0; m < q.m && identity; m++) identity = q.cperm[m] == m;
    // One part unless forced: on B200 at N = 1e5, M = 1e6 (CS 128 MB per group) the
    // split did not pay -- 57.5k RHS/s in one part, 51.0k in two, 43.9k in four: the
    // extra launches cost more than the L2 hits save.
    int parts = 1;
    if (identity && s->stream_parts > 0) parts = std::min(s->stream_parts, std::max(1, q.m));
    std::vector<int> start(q.n + 1, 0), deg(q.n, 0);
    for (int qq = 0; qq < q.k; qq++)
        for (int m = 0; m < q.m; m++) {
            const uint32_t v = q.litw[(size_t)qq * q.mp + m] & 0x7fffffffu;
            if ((int)v < q.n) deg[v]++;
        }
    for (int v = 0; v < q.n; v++) start[v + 1] = start[v] + deg[v];
    std::vector<int> pos(std::max(start[q.n], 1), 0);
    for (int qq = 0; qq < q.k; qq++)
        for (int m = 0; m < q.m; m++) {
            const size_t idx = (size_t)qq * q.mp + m;
            const uint32_t v = q.litw[idx] & 0x7fffffffu;
            if ((int)v >= q.n) continue;
            const int rank = (int)(q.slotw[idx] >> 5) - q.srow[v >> 5];  // row in v's SELL list
            pos[start[v] + rank] = (int)idx;
        }
    std::vector<int> split((size_t)(parts + 1) * q.n);
    for (int v = 0; v < q.n; v++) {
        int r = start[v];
        for (int pp = 0; pp < parts; pp++) {
            split[(size_t)pp * q.n + v] = r;
            const long long m1 = (long long)q.m * (pp + 1) / parts;
            while (r < start[v + 1] && (pos[r] % q.mp) < m1) r++;
        }
        split[(size_t)parts * q.n + v] = start[v + 1];
    }
    P.vstart[p].reset(new DevBuf());
    P.vpos[p].reset(new DevBuf());
    AS_CUDA(P.vstart[p]->alloc(sizeof(int) * std::max<size_t>(split.size(), 1)));
    AS_CUDA(P.vpos[p]->alloc(sizeof(int) * pos.size()));
    if (!split.empty())
        AS_CUDA(cudaMemcpy(P.vstart[p]->p, split.data(), sizeof(int) * split.size(), cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemcpy(P.vpos[p]->p, pos.data(), sizeof(int) * pos.size(), cudaMemcpyHostToDevice));
    P.nparts[p] = parts;
    P.have_lists[p] = 1;
    return AS_OK;
}

// Units sorted by problem, groups of four lanes, device storage and lane states.
int stream_plan(as_solver* s) {
    const int num_traj = s->num_traj;
    const auto& pi = s->traj_problem;
    s->order.resize(num_traj);
    for (int t = 0; t < num_traj; t++) s->order[t] = t;
    std::stable_sort(s->order.begin(), s->order.end(), [&](int a, int b) { return pi[a] < pi[b]; });
    if (!s->sp) s->sp.reset(new StreamPlan());
    StreamPlan& P = *s->sp;
    P.gprob.clear();
    P.goff.clear();
    P.gcand.clear();
    std::vector<LaneState> lanes;
    const size_t vbytes = s->precision == AS_PREC_F64 ? 8 : 4;
    size_t total = 0, cand_words = 0;
    for (int u = 0; u < num_traj;) {
        const int p = pi[s->order[u]];
        const auto& q = s->problems[p];
        P.gprob.push_back(p);
        P.goff.push_back(total);
        P.gcand.push_back(cand_words);
        total += stream_group_bytes(q, vbytes);
        cand_words += (size_t)kLanes * ((q.n + 31) / 32);
        for (int l = 0; l < kLanes; l++) {
            LaneState L;
            std::memset(&L, 0, sizeof(L));
            L.h = L.h0 = L.hnext = 1e-9;  // CpuRungeKutta's first step (as solve_kernel)
            L.viol = -1;
            L.minviol = INT_MAX;
            L.unit = -1;
            L.status = -1;  // padding lane: never runs
            if (u < num_traj && pi[s->order[u]] == p) {
                L.unit = u;
                if (0.0 < s->max_time && 0 < s->max_steps) {
                    L.status = SAT_UNKNOWN;
                    L.rhs = 1;  // k1 of the first step
                } else {
                    L.status = 0.0 >= s->max_time ? SAT_MAXTIME_REACHED : SAT_MAXITER_REACHED;
                }
                u++;
            }
            lanes.push_back(L);
        }
    }
    P.ngroups = (int)P.gprob.size();
    const size_t np = s->problems.size();
    if (P.have_lists.size() != np) {
        P.have_lists.assign(np, 0);
        P.nparts.assign(np, 1);
        P.vstart.resize(np);
        P.vpos.resize(np);
    }
    for (int p : P.gprob)
        if (!P.have_lists[p]) {
            int r = stream_lists(s, p);
            if (r) return r;
        }
    AS_CUDA(P.vec.alloc(std::max<size_t>(total, 256)));
    AS_CUDA(P.lanes.alloc(sizeof(LaneState) * lanes.size()));
    AS_CUDA(P.tickets.alloc(sizeof(int) * 2 * P.ngroups));
    AS_CUDA(P.active.alloc(sizeof(int) * P.ngroups));
    AS_CUDA(P.cand.alloc(sizeof(uint32_t) * std::max<size_t>(cand_words, 1)));
    std::vector<int> act(P.ngroups, 0);
    for (int g = 0; g < P.ngroups; g++)
        for (int l = 0; l < kLanes; l++) act[g] += lanes[(size_t)g * kLanes + l].status == SAT_UNKNOWN;
    std::vector<int> ui(num_traj);
    std::vector<long long> us(num_traj), ub(num_traj);
    for (int u = 0; u < num_traj; u++) {
        ui[u] = pi[s->order[u]];
        us[u] = s->traj_off[s->order[u]];
        ub[u] = s->traj_bits[s->order[u]];
    }
    AS_CUDA(cudaMemcpy(P.lanes.p, lanes.data(), sizeof(LaneState) * lanes.size(), cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemcpy(P.active.p, act.data(), sizeof(int) * P.ngroups, cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemset(P.tickets.p, 0, sizeof(int) * 2 * P.ngroups));
    AS_CUDA(cudaMemcpy(s->unit_inst.p, ui.data(), sizeof(int) * num_traj, cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemcpy(s->unit_state.p, us.data(), sizeof(long long) * num_traj, cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemcpy(s->unit_bits.p, ub.data(), sizeof(long long) * num_traj, cudaMemcpyHostToDevice));
    return AS_OK;
}

// One pass (an RK attempt of every lane) of every group, in stream order.
template <typename T, bool LOGA, int KMAX, bool EXACT>
int stream_record_pass(as_solver* s, cudaStream_t st, const unsigned long long* deadline) {
    StreamPlan& P = *s->sp;
    constexpr int BT = 256;
    const int sms = s->sm_count;
    for (int g = 0; g < P.ngroups; g++) {
        StreamArgs<T> A = stream_args<T>(s, g, deadline);
        const int n = A.I.n, m = A.I.m;
        // kRowThreads threads per clause / variable row in the stage kernels
        const int gc = (int)std::max(1ll, std::min(((long long)kRowThreads * m + BT - 1) / BT, (long long)sms * 8));
        const int gv = (int)std::max(1ll, std::min(((long long)kRowThreads * n + BT - 1) / BT, (long long)sms * 8));
        const int* vstart0 = A.vstart;
        for (int S = 1; S <= 6; S++) {
            A.S = S;
            for (int part = 0; part < A.nparts; part++) {
                A.part = part;
                A.m0 = (int)((long long)m * part / A.nparts);
                A.m1 = (int)((long long)m * (part + 1) / A.nparts);
                A.vstart = vstart0 + (size_t)part * n;
                const int gcp = (int)std::max(1ll, std::min(((long long)kRowThreads * (A.m1 - A.m0) + BT - 1) / BT,
                                                            (long long)sms * 8));
                stream_clause_kernel<T, LOGA, KMAX, EXACT><<<gcp, BT, 0, st>>>(A);
                stream_var_kernel<T, LOGA><<<gv, BT, 0, st>>>(A);
            }
        }
        A.vstart = vstart0;
        A.part = 0;
        const int words = (n + 31) / 32;
        const int nbw = s->track_best ? std::max(1, std::min((words + BT / 32 - 1) / (BT / 32), sms * 2)) : 0;
        const int pv = std::max(1, std::min((n + BT - 1) / BT, sms * 4));
        const int pc = std::max(1, std::min((m + BT - 1) / BT, sms * 8));
        stream_post_kernel<T, KMAX, EXACT><<<pv + pc + nbw, BT, 0, st>>>(A, pv, pc);
        s->last_bt = BT;
        s->last_kernel = "stream_clause_kernel+stream_var_kernel";
        s->last_ctas = gc;
        s->last_smem = 0;
        s->last_occ = 0;
    }
    AS_CUDA(cudaGetLastError());
    return AS_OK;
}

template <typename T, bool LOGA, int KMAX, bool EXACT>
int stream_run(as_solver* s) {
    StreamPlan& P = *s->sp;
    cudaStream_t st = s->stream;
    AS_CUDA(cudaMemsetAsync(s->solved.p, 0, s->solved.bytes, st));
    const bool have_deadline = s->wall_budget > 0.0;
    const unsigned long long* deadline = have_deadline ? s->deadline.as<unsigned long long>() : nullptr;
    if (have_deadline) {
        stamp_deadline_kernel<<<1, 1, 0, st>>>(s->deadline.as<unsigned long long>(),
                                               (unsigned long long)(s->wall_budget * 1e9));
        AS_CUDA(cudaGetLastError());
    }
    for (int g = 0; g < P.ngroups; g++) {
        StreamArgs<T> A = stream_args<T>(s, g, deadline);
        const long long E = (long long)A.I.n + A.I.m;
        const int blocks = (int)std::max(1ll, std::min((E + 255) / 256, (long long)s->sm_count * 8));
        stream_load_kernel<T, LOGA><<<blocks, 256, 0, st>>>(A, static_cast<const T*>(s->states.p),
                                                            s->unit_state.as<long long>());
    }
    AS_CUDA(cudaGetLastError());
    if (P.graph) { cudaGraphExecDestroy(P.graph); P.graph = nullptr; }
    cudaGraph_t graph = nullptr;
    AS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int r = stream_record_pass<T, LOGA, KMAX, EXACT>(s, st, deadline);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (r) { if (graph) cudaGraphDestroy(graph); return r; }
    if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("stream graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&P.graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("stream graph instantiate: ") + cudaGetErrorString(e));
    // Passes until every lane has finished.  The device applies the status rules and
    // the wall-clock deadline (at every attempt); the host only polls the active-lane
    // counts between chunks of passes.
    std::vector<int> act(P.ngroups);
    P.passes = 0;
    int chunk = 2;
    while (true) {
        for (int i = 0; i < chunk; i++) AS_CUDA(cudaGraphLaunch(P.graph, st));
        P.passes += chunk;
        AS_CUDA(cudaMemcpyAsync(act.data(), P.active.p, sizeof(int) * P.ngroups, cudaMemcpyDeviceToHost, st));
        AS_CUDA(cudaStreamSynchronize(st));
        bool any = false;
        for (int a : act) any |= a != 0;
        if (!any) break;
        chunk = std::min(chunk * 2, 16);
    }
    for (int g = 0; g < P.ngroups; g++) {
        StreamArgs<T> A = stream_args<T>(s, g, deadline);
        const long long E = (long long)A.I.n + A.I.m;
        const int blocks = (int)std::max(1ll, std::min((E + 255) / 256, (long long)s->sm_count * 8));
        stream_store_kernel<T, LOGA><<<blocks, 256, 0, st>>>(A, static_cast<T*>(s->states.p),
                                                             s->unit_state.as<long long>(),
                                                             s->results.as<UnitResult>());
    }
    AS_CUDA(cudaGetLastError());
    AS_CUDA(cudaStreamSynchronize(st));
    return AS_OK;
}

int stream_solve(as_solver* s) {
    for (const auto& q : s->problems)
        if (!standard_model(q))
            return fail(AS_ERR_UNSUPPORTED, "the streamed solver has the plain CTDS right-hand side only "
                                            "(no tanh variant, no bias term)");
    int r = stream_plan(s);
    if (r) return r;
    bool all3 = true, all4 = true;
    int kmax = 0;
    for (int p : s->sp->gprob) {
        kmax = std::max(kmax, s->problems[p].k);
        all3 = all3 && s->problems[p].k == 3;
        all4 = all4 && s->problems[p].k == 4;
    }
    if (kmax > 16) return fail(AS_ERR_UNSUPPORTED, "clause length > 16 is not supported");
    if (s->precision == AS_PREC_F64) {
        if (all3) return stream_run<double, false, 3, true>(s);
        if (all4) return stream_run<double, false, 4, true>(s);
        return stream_run<double, false, 16, false>(s);
    }
    if (all3) return stream_run<float, true, 3, true>(s);
    if (all4) return stream_run<float, true, 4, true>(s);
    return stream_run<float, true, 16, false>(s);
}

}  // namespace

int32_t as_solver_set_states_f64(as_solver* s, const int32_t* pi, int32_t nt, const double* st) {
    return set_states_host<double>(s, pi, nt, st);
}
int32_t as_solver_set_states_f32(as_solver* s, const int32_t* pi, int32_t nt, const float* st) {
    return set_states_host<float>(s, pi, nt, st);
}
int32_t as_solver_set_states_device(as_solver* s, const int32_t* pi, int32_t nt, const void* src,
                                    void* stream) {
    if (!s || !src) return fail(AS_ERR_BAD_INPUT, "as_solver_set_states_device: null argument");
    AS_CUDA(cudaSetDevice(s->device));
    int r = plan_units(s, pi, nt);
    if (r) return r;
    const size_t vb = s->precision == AS_PREC_F64 ? 8 : 4;
    AS_CUDA(cudaMemcpyAsync(s->states.p, src, (size_t)s->total_values * vb, cudaMemcpyDeviceToDevice,
                            stream ? (cudaStream_t)stream : s->stream));
    if (stream) AS_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return AS_OK;
}

int32_t as_solver_set_random_states(as_solver* s, const int32_t* pi, int32_t nt, uint64_t seed,
                                    int32_t distribution, double a0) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "as_solver_set_random_states: null solver");
    if (distribution != AS_IC_SPIN_UNIFORM && distribution != AS_IC_REFERENCE)
        return fail(AS_ERR_BAD_INPUT, "as_solver_set_random_states: unknown distribution");
    if (distribution == AS_IC_SPIN_UNIFORM && !(a0 > 0.0 && std::isfinite(a0)))
        return fail(AS_ERR_BAD_INPUT, "as_solver_set_random_states: need a0 > 0");
    AS_CUDA(cudaSetDevice(s->device));
    int r = plan_units(s, pi, nt);
    if (r) return r;
    std::vector<asb::IcTraj> tr(nt);
    for (int t = 0; t < nt; t++) {
        const auto& q = s->problems[pi[t]];
        tr[t] = asb::IcTraj{s->traj_off[t], q.n, q.m};
    }
    const cudaError_t e = asb::random_states(s->states.p, s->precision == AS_PREC_F64, tr, seed, distribution, a0,
                                            s->stream);
    if (e != cudaSuccess)
        return fail(AS_ERR_CUDA, std::string("as_solver_set_random_states: ") + cudaGetErrorString(e));
    return AS_OK;
}

int32_t as_solver_solve_async(as_solver* s, void* stream) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (s->num_traj <= 0) return fail(AS_ERR_NO_PROBLEM, "no trajectories set (as_solver_set_states_*)");
    AS_CUDA(cudaSetDevice(s->device));
    if (use_stream(s)) {  // host-driven passes: runs to completion on the solver's stream
        if (stream && (cudaStream_t)stream != s->stream) AS_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
        AS_CUDA(cudaStreamSynchronize(s->stream));
        s->groups_dirty = true;
        return stream_solve(s);
    }
    if (s->groups_dirty) {
        int r = build_groups(s);
        if (r) return r;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    if (st != s->stream) {
        // The solve runs on the caller's stream: after the work already queued on the
        // solver's stream (states copied in by as_solver_set_states_*), and before
        // anything queued there later (as_solver_sync, result and state reads).
        if (!s->ev_in) AS_CUDA(cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming));
        if (!s->ev_out) AS_CUDA(cudaEventCreateWithFlags(&s->ev_out, cudaEventDisableTiming));
        AS_CUDA(cudaEventRecord(s->ev_in, s->stream));
        AS_CUDA(cudaStreamWaitEvent(st, s->ev_in, 0));
        int r = record_solve(s, st);
        if (r) return r;
        AS_CUDA(cudaEventRecord(s->ev_out, st));
        AS_CUDA(cudaStreamWaitEvent(s->stream, s->ev_out, 0));
        return AS_OK;
    }
    if (!s->graph_valid) {
        if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
        cudaGraph_t g = nullptr;
        AS_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        int r = record_solve(s, s->stream);
        cudaError_t e = cudaStreamEndCapture(s->stream, &g);
        if (r) { if (g) cudaGraphDestroy(g); return r; }
        if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&s->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        s->graph_valid = true;
    }
    AS_CUDA(cudaGraphLaunch(s->graph, s->stream));
    return AS_OK;
}

int32_t as_solver_sync(as_solver* s) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    AS_CUDA(cudaStreamSynchronize(s->stream));
    return AS_OK;
}

int32_t as_solver_solve(as_solver* s) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    const auto w0 = std::chrono::steady_clock::now();
    const std::clock_t c0 = std::clock();
    int r = as_solver_solve_async(s, nullptr);
    if (!r) r = as_solver_sync(s);
    s->last_wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    s->last_cpu = (double)(std::clock() - c0) / CLOCKS_PER_SEC;
    return r;
}

const char* as_result_message(int32_t result) {
    switch (result) {  // GetSatResultMessage (AnalogSAT/solver/SatResult.cpp)
        case SAT_SOLUTION_FOUND: return "solution found";
        case SAT_UNDERFLOW: return "underflow";
        case SAT_ODE_INTERRUPTED: return "user interrupt";
        case SAT_MAXTIME_REACHED: return "maximum time reached";
        case SAT_MAXITER_REACHED: return "maximum steps reached";
        default: return "unknown result";
    }
}

int32_t as_solver_write_result(as_solver* s, int32_t traj, const char* path) {
    if (!s || !path) return fail(AS_ERR_BAD_INPUT, "as_solver_write_result: null argument");
    if (traj < 0 || traj >= s->num_traj) return fail(AS_ERR_BAD_INPUT, "trajectory index out of range");
    std::vector<int32_t> status(s->num_traj);
    int r = as_solver_get_results(s, status.data(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (r) return r;
    const int n = s->problems[s->traj_problem[traj]].n;
    std::vector<double> x((size_t)s->total_values);
    r = as_solver_get_states_f64(s, x.data());
    if (r) return r;
    const double* st = x.data() + s->traj_off[traj];
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(AS_ERR_IO, std::string("cannot open result file to write: ") + path);
    // MiniSat-compatible: SAT or INDET (an incomplete solver cannot prove UNSAT), then
    // the assignment as signed variable numbers terminated by 0 (cnf_runner.cpp:280-304)
    std::fprintf(f, "%s\n", status[traj] == SAT_SOLUTION_FOUND ? "SAT" : "INDET");
    if (n > 0) std::fprintf(f, "%d", st[0] > 0 ? 1 : -1);
    for (int i = 1; i < n; i++) std::fprintf(f, " %d", st[i] > 0.0 ? i + 1 : -i - 1);
    std::fprintf(f, " 0\n");
    const bool ok = std::fclose(f) == 0;
    return ok ? AS_OK : fail(AS_ERR_IO, std::string("cannot write ") + path);
}

int32_t as_solver_append_perf(as_solver* s, int32_t traj, const char* path, const char* sample,
                              const char* solver_name) {
    if (!s || !path || !sample || !solver_name) return fail(AS_ERR_BAD_INPUT, "as_solver_append_perf: null argument");
    if (traj < 0 || traj >= s->num_traj) return fail(AS_ERR_BAD_INPUT, "trajectory index out of range");
    std::vector<int32_t> status(s->num_traj), rhs(s->num_traj);
    int r = as_solver_get_results(s, status.data(), nullptr, nullptr, rhs.data(), nullptr, nullptr, nullptr, nullptr);
    if (r) return r;
    cudaDeviceProp prop;
    AS_CUDA(cudaGetDeviceProperties(&prop, s->device));
    FILE* f = std::fopen(path, "a");
    if (!f) return fail(AS_ERR_IO, std::string("cannot open ") + path);
    // sample, GPU, solver, answer, wall time, CPU time, RHS count (bench_runner.cpp:331-343)
    std::fprintf(f, "%s\t%s\t%s\t%s\t%lf\t%lf\t%d\n", sample, prop.name, solver_name,
                 as_result_message(status[traj]), s->last_wall, s->last_cpu, rhs[traj]);
    const bool ok = std::fclose(f) == 0;
    return ok ? AS_OK : fail(AS_ERR_IO, std::string("cannot write ") + path);
}

int32_t as_solver_get_results(as_solver* s, int32_t* status, double* time, int32_t* steps, int32_t* rhs,
                              int32_t* attempts, int32_t* violations, int32_t* min_violations,
                              double* last_step) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (s->num_traj <= 0) return fail(AS_ERR_NO_PROBLEM, "no trajectories set");
    std::vector<UnitResult> r(s->num_traj);
    AS_CUDA(cudaSetDevice(s->device));
    AS_CUDA(cudaMemcpyAsync(r.data(), s->results.p, sizeof(UnitResult) * s->num_traj, cudaMemcpyDeviceToHost,
                            s->stream));
    AS_CUDA(cudaStreamSynchronize(s->stream));
    for (int u = 0; u < s->num_traj; u++) {
        const int t = s->order[u];
        if (status) status[t] = r[u].status;
        if (time) time[t] = r[u].time;
        if (steps) steps[t] = r[u].steps;
        if (rhs) rhs[t] = r[u].rhs;
        if (attempts) attempts[t] = r[u].attempts;
        if (violations) violations[t] = r[u].viol;
        if (min_violations) min_violations[t] = r[u].min_viol;
        if (last_step) last_step[t] = r[u].hdid;
    }
    return AS_OK;
}

namespace {
template <typename DST>
int get_states(as_solver* s, DST* out) {
    if (!s || !out) return fail(AS_ERR_BAD_INPUT, "as_solver_get_states: null argument");
    if (s->num_traj <= 0) return fail(AS_ERR_NO_PROBLEM, "no trajectories set");
    AS_CUDA(cudaSetDevice(s->device));
    const size_t n = (size_t)s->total_values;
    const size_t vb = s->precision == AS_PREC_F64 ? 8 : 4;
    if (vb == sizeof(DST)) {
        AS_CUDA(cudaMemcpyAsync(out, s->states.p, n * vb, cudaMemcpyDeviceToHost, s->stream));
        AS_CUDA(cudaStreamSynchronize(s->stream));
    } else if (vb == 8) {
        std::vector<double> tmp(n);
        AS_CUDA(cudaMemcpyAsync(tmp.data(), s->states.p, n * 8, cudaMemcpyDeviceToHost, s->stream));
        AS_CUDA(cudaStreamSynchronize(s->stream));
        for (size_t i = 0; i < n; i++) out[i] = (DST)tmp[i];
    } else {
        std::vector<float> tmp(n);
        AS_CUDA(cudaMemcpyAsync(tmp.data(), s->states.p, n * 4, cudaMemcpyDeviceToHost, s->stream));
        AS_CUDA(cudaStreamSynchronize(s->stream));
        for (size_t i = 0; i < n; i++) out[i] = (DST)tmp[i];
    }
    return AS_OK;
}
}  // namespace

template <typename DST>
int get_state_one(as_solver* s, int32_t traj, DST* out) {
    if (!s || !out) return fail(AS_ERR_BAD_INPUT, "as_solver_get_state: null argument");
    if (traj < 0 || traj >= s->num_traj) return fail(AS_ERR_BAD_INPUT, "trajectory index out of range");
    AS_CUDA(cudaSetDevice(s->device));
    const auto& q = s->problems[s->traj_problem[traj]];
    const size_t n = (size_t)q.n + q.m;
    const size_t vb = s->precision == AS_PREC_F64 ? 8 : 4;
    const char* src = static_cast<const char*>(s->states.p) + (size_t)s->traj_off[traj] * vb;
    if (vb == sizeof(DST)) {
        AS_CUDA(cudaMemcpyAsync(out, src, n * vb, cudaMemcpyDeviceToHost, s->stream));
        AS_CUDA(cudaStreamSynchronize(s->stream));
    } else if (vb == 8) {
        std::vector<double> tmp(n);
        AS_CUDA(cudaMemcpyAsync(tmp.data(), src, n * 8, cudaMemcpyDeviceToHost, s->stream));
        AS_CUDA(cudaStreamSynchronize(s->stream));
        for (size_t i = 0; i < n; i++) out[i] = (DST)tmp[i];
    } else {
        std::vector<float> tmp(n);
        AS_CUDA(cudaMemcpyAsync(tmp.data(), src, n * 4, cudaMemcpyDeviceToHost, s->stream));
        AS_CUDA(cudaStreamSynchronize(s->stream));
        for (size_t i = 0; i < n; i++) out[i] = (DST)tmp[i];
    }
    return AS_OK;
}

int32_t as_solver_get_states_f64(as_solver* s, double* out) { return get_states<double>(s, out); }
int32_t as_solver_get_state_f64(as_solver* s, int32_t traj, double* out) { return get_state_one<double>(s, traj, out); }
int32_t as_solver_get_state_f32(as_solver* s, int32_t traj, float* out) { return get_state_one<float>(s, traj, out); }
int32_t as_solver_get_states_f32(as_solver* s, float* out) { return get_states<float>(s, out); }
const void* as_solver_states_device(as_solver* s) { return s ? s->states.p : nullptr; }

int32_t as_solver_get_best_assignment(as_solver* s, int32_t traj, uint32_t* bits) {
    if (!s || !bits) return fail(AS_ERR_BAD_INPUT, "as_solver_get_best_assignment: null argument");
    if (traj < 0 || traj >= s->num_traj) return fail(AS_ERR_BAD_INPUT, "trajectory index out of range");
    if (!s->track_best) return fail(AS_ERR_BAD_INPUT, "best-assignment tracking is off");
    const auto& q = s->problems[s->traj_problem[traj]];
    AS_CUDA(cudaSetDevice(s->device));
    AS_CUDA(cudaMemcpyAsync(bits, s->best_bits.as<uint32_t>() + s->traj_bits[traj],
                            sizeof(uint32_t) * ((q.n + 31) / 32), cudaMemcpyDeviceToHost, s->stream));
    AS_CUDA(cudaStreamSynchronize(s->stream));
    return AS_OK;
}

int32_t as_solver_get_launch_shape(as_solver* s, int32_t* threads, int32_t* ctas, int32_t* smem_bytes,
                                   int32_t* ctas_per_sm) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (threads) *threads = s->last_bt;
    if (ctas) *ctas = s->last_ctas;
    if (smem_bytes) *smem_bytes = s->last_smem;
    if (ctas_per_sm) *ctas_per_sm = s->last_occ;
    return AS_OK;
}

int32_t as_solver_set_storage_mode(as_solver* s, int32_t mode) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (mode < 0 || mode > 3) return fail(AS_ERR_BAD_INPUT, "storage mode must be 0, 1, 2 or 3");
    s->storage_mode = mode;
    s->groups_dirty = true;
    s->invalidate();
    return AS_OK;
}

int32_t as_solver_set_stream_parts(as_solver* s, int32_t parts) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (parts < 0 || parts > 8) return fail(AS_ERR_BAD_INPUT, "stream parts must be 0 (automatic) to 8");
    s->stream_parts = parts;
    if (s->sp) s->sp->have_lists.clear();
    return AS_OK;
}

int32_t as_solver_set_cluster_size(as_solver* s, int32_t ctas) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (!(ctas == 0 || ctas == 1 || ctas == 4 || ctas == 8))
        return fail(AS_ERR_BAD_INPUT, "cluster size must be 0 (automatic), 1, 4 or 8");
    s->forced_cl = ctas;
    s->groups_dirty = true;
    s->invalidate();
    return AS_OK;
}

const char* as_solver_kernel_name(const as_solver* s) { return s ? s->last_kernel : ""; }

int32_t as_solver_set_kernel(as_solver* s, int32_t kernel) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (kernel != AS_KERNEL_AUTO && kernel != AS_KERNEL_GENERIC)
        return fail(AS_ERR_BAD_INPUT, "as_solver_set_kernel: AS_KERNEL_AUTO or AS_KERNEL_GENERIC");
    s->kernel_choice = kernel;
    s->groups_dirty = true;
    s->invalidate();
    return AS_OK;
}

int32_t as_solver_force_threads(as_solver* s, int32_t threads) {
    if (!s) return fail(AS_ERR_BAD_INPUT, "null solver");
    if (threads != 0 && (threads < 32 || threads > 1024 || threads % 32 != 0))
        return fail(AS_ERR_BAD_INPUT, "CTA size must be a multiple of 32 in [32, 1024]");
    s->forced_bt = threads;
    s->groups_dirty = true;
    s->invalidate();
    return AS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free solve (as_solver_solve_noalloc)
//
// For callers that must not allocate device memory once they are running -- for
// example an application that reserves all of the GPU's memory up front for its own
// pool, or a fixed-latency loop in which a cudaMalloc (which can synchronise the
// device) is not allowed.  The per-call scratch of the persistent solve kernel (the
// work counter, the instance's first-solution flag, the wall-clock deadline and the
// trajectory tables) lives in the file-scope array below instead of in buffers owned
// by the solver handle.  The array is part of the library image: every GPU that
// loads the library holds its AS_NOALLOC_SCRATCH_BYTES until the process exits.
// Every call shares it; each call re-initialises it, so two calls whose kernels
// overlap on the GPU (different streams, or different host threads) race.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocFlags = AS_NOALLOC_MAX_PROBLEM_INDEX;
constexpr size_t kNoAllocHeader = 256;  // work counter + deadline, padded
constexpr size_t kNoAllocFlagBytes = sizeof(int) * kNoAllocFlags;
constexpr size_t kNoAllocInstOff = kNoAllocHeader + kNoAllocFlagBytes;
constexpr size_t kNoAllocStateOff = kNoAllocInstOff + sizeof(int) * AS_NOALLOC_MAX_TRAJ;
constexpr size_t kNoAllocBytes = kNoAllocStateOff + sizeof(long long) * AS_NOALLOC_MAX_TRAJ;
static_assert(kNoAllocBytes == AS_NOALLOC_SCRATCH_BYTES, "scratch size documented in the header");
static_assert(kNoAllocInstOff % 16 == 0 && kNoAllocStateOff % 16 == 0, "scratch alignment");
static_assert(sizeof(as_unit_result) == sizeof(UnitResult), "as_unit_result mirrors UnitResult");
static_assert(offsetof(as_unit_result, status) == offsetof(UnitResult, status), "layout");
static_assert(offsetof(as_unit_result, min_violations) == offsetof(UnitResult, min_viol), "layout");

static __device__ __align__(256) unsigned char as_noalloc_scratch[kNoAllocBytes];

// Device address of the scratch array per device (host code only sees a host-side
// stand-in for the symbol; the address comes from cudaGetSymbolAddress).
std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {};

int noalloc_scratch_address(int dev, unsigned char** out) {
    if (dev < 0 || dev >= 256) return fail(AS_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, as_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(AS_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[dev]);
    return AS_OK;
}

// Resets the per-call words (work counter, this instance's flag, deadline) and writes
// the trajectory tables: trajectory u solves problem pidx from states + u * stride.
__global__ void noalloc_prepare_kernel(unsigned char* scratch, int pidx, int num_traj,
                                       long long stride, unsigned long long budget_ns) {
    int* head = reinterpret_cast<int*>(scratch);
    unsigned long long* deadline = reinterpret_cast<unsigned long long*>(scratch + 8);
    int* flags = reinterpret_cast<int*>(scratch + kNoAllocHeader);
    int* inst = reinterpret_cast<int*>(scratch + kNoAllocInstOff);
    long long* off = reinterpret_cast<long long*>(scratch + kNoAllocStateOff);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        *head = 0;
        flags[pidx] = 0;
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        *deadline = t + budget_ns;
    }
    for (int u = i; u < num_traj; u += gridDim.x * blockDim.x) {
        inst[u] = pidx;
        off[u] = (long long)u * stride;
    }
}

}  // namespace

int32_t as_solver_solve_noalloc(as_solver* s, int32_t problem_index, int32_t num_traj, void* states,
                                as_unit_result* results, void* stream) {
    if (!s || !states || !results) return fail(AS_ERR_BAD_INPUT, "as_solver_solve_noalloc: null argument");
    if (problem_index < 0 || problem_index >= (int)s->problems.size())
        return fail(AS_ERR_BAD_INPUT, "as_solver_solve_noalloc: problem index out of range");
    if (problem_index >= AS_NOALLOC_MAX_PROBLEM_INDEX)
        return fail(AS_ERR_UNSUPPORTED, "as_solver_solve_noalloc: problem index must be < "
                                        "AS_NOALLOC_MAX_PROBLEM_INDEX (4096)");
    if (num_traj < 1 || num_traj > AS_NOALLOC_MAX_TRAJ)
        return fail(AS_ERR_UNSUPPORTED, "as_solver_solve_noalloc: num_traj must be in [1, "
                                        "AS_NOALLOC_MAX_TRAJ] (65536)");
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    unsigned char* scratch = nullptr;
    int r = noalloc_scratch_address(s->device, &scratch);
    if (r) return r;

    const PackedProblem& q = s->problems[problem_index];
    const Variant* v = nullptr;
    long best = -1;
    for (const auto& cand : variants()) {
        if (cand.gs || !fits(cand, q, s->precision, s->smem_limit)) continue;
        if (cand.lean && s->kernel_choice == AS_KERNEL_GENERIC) continue;
        const long score = variant_score(cand);
        if (!v || score < best) { best = score; v = &cand; }
    }
    if (!v)
        return fail(AS_ERR_UNSUPPORTED, "as_solver_solve_noalloc: the instance does not fit one SM's shared "
                                        "memory (only shared-memory launches need no device buffers)");
    int bt = s->forced_bt;
    if (!bt) {
        r = shared_cta_threads(solver_smem(*v, q), std::max(64, preferred_bt(q)), s->device, &bt);
        if (r) return r;
    }
    const size_t smem = solver_smem(*v, q);
    cudaStream_t st = (cudaStream_t)stream;

    noalloc_prepare_kernel<<<std::max(1, std::min(s->sm_count, (num_traj + 255) / 256)), 256, 0, st>>>(
        scratch, problem_index, num_traj, (long long)(q.n + q.m),
        s->wall_budget > 0.0 ? (unsigned long long)(s->wall_budget * 1e9) : 0ull);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("prepare launch: ") + cudaGetErrorString(e));
    e = raise_smem_limit((const void*)v->fn, smem);
    if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v->fn, bt, smem);
    if (e != cudaSuccess || occ < 1) return fail(AS_ERR_UNSUPPORTED, "launch shape does not fit on an SM");

    SolveParams P;
    P.inst = s->pool.inst.as<DevInstance>();
    P.unit_inst = reinterpret_cast<const int*>(scratch + kNoAllocInstOff);
    P.unit_state = reinterpret_cast<const long long*>(scratch + kNoAllocStateOff);
    P.states = states;
    P.results = reinterpret_cast<UnitResult*>(results);
    P.queue_head = reinterpret_cast<int*>(scratch);
    P.inst_solved = reinterpret_cast<int*>(scratch + kNoAllocHeader);
    P.best_bits = nullptr;
    P.unit_bits = nullptr;
    P.num_units = num_traj;
    P.maxsteps = s->max_steps;
    P.batch = s->batch;
    P.stop_on_first = s->stop_on_first;
    P.eps = s->eps;
    P.tmax = s->max_time;
    P.deadline = s->wall_budget > 0.0 ? reinterpret_cast<const unsigned long long*>(scratch + 8) : nullptr;
    P.slab = nullptr;
    P.slab_stride = 0;
    void* args[] = {&P};
    e = cudaLaunchKernel((const void*)v->fn, dim3(std::min(num_traj, s->sm_count * occ)), dim3(bt), args,
                         smem, st);
    if (e != cudaSuccess) return fail(AS_ERR_CUDA, std::string("solve launch: ") + cudaGetErrorString(e));
    return AS_OK;
}

// ---------------------------------------------------------------------------
// Adjoint (gradients of the final potential)
// ---------------------------------------------------------------------------
#include "as_adjoint.cuh"

namespace {

using AdjFn = void (*)(AdjointParams);

struct AdjVariant {
    int precision, kmax;
    bool exact;
    AdjFn fwd, bwd;
    size_t bytes;
};

#define AS_ADJ(T, P, K, EX) \
    AdjVariant{P, K, EX, &adj_forward_kernel<T, K, EX>, &adj_backward_kernel<T, K, EX>, sizeof(T)}

const std::vector<AdjVariant>& adj_variants() {
    static const std::vector<AdjVariant> v = {
        AS_ADJ(float, AS_PREC_F32_LOGA, 3, true),  AS_ADJ(float, AS_PREC_F32_LOGA, 16, false),
        AS_ADJ(double, AS_PREC_F64, 3, true),      AS_ADJ(double, AS_PREC_F64, 16, false),
    };
    return v;
}

}  // namespace

int32_t as_solver_adjoint(as_solver* s, double t_end, int32_t max_steps, const double* weights, double* loss,
                          double* grad_x0, double* grad_w, int32_t* nsteps, double* step_sizes) {
    if (!s || !loss || !grad_x0 || !grad_w) return fail(AS_ERR_BAD_INPUT, "as_solver_adjoint: null argument");
    if (!(t_end > 0.0) || max_steps < 1) return fail(AS_ERR_BAD_INPUT, "as_solver_adjoint: need t_end > 0, max_steps >= 1");
    if (s->num_traj <= 0) return fail(AS_ERR_NO_PROBLEM, "no trajectories set (as_solver_set_states_*)");
    for (const auto& q : s->problems)
        if (!standard_model(q))
            return fail(AS_ERR_UNSUPPORTED, "the adjoint covers the plain CTDS right-hand side only");
    AS_CUDA(cudaSetDevice(s->device));
    const int nt = s->num_traj;
    // one launch shape for all trajectories: the largest instance decides
    const AdjVariant* av = nullptr;
    size_t vals = 0;
    int bt = 64;
    for (int t = 0; t < nt; t++) {
        const auto& q = s->problems[s->traj_problem[t]];
        if (!q.compact) return fail(AS_ERR_UNSUPPORTED, "adjoint: instance beyond the compact encoding");
        vals = std::max(vals, adjoint_smem_values(q.n, q.m, q.nslots));
        bt = std::max(bt, preferred_bt(q));
    }
    for (const auto& v : adj_variants()) {
        bool ok = v.precision == s->precision;
        for (int t = 0; ok && t < nt; t++) {
            const int k = s->problems[s->traj_problem[t]].k;
            ok = v.exact ? k == v.kmax : k <= v.kmax;
        }
        if (ok) { av = &v; break; }
    }
    if (!av) return fail(AS_ERR_UNSUPPORTED, "adjoint: clause length > 16");
    const size_t smem = vals * av->bytes;
    if (smem > s->smem_limit) return fail(AS_ERR_UNSUPPORTED, "adjoint: instance too large for one SM");

    std::vector<int> ui(nt);
    std::vector<long long> us(nt), uw(nt);
    long long wtot = 0;
    for (int t = 0; t < nt; t++) {
        ui[t] = s->traj_problem[t];
        us[t] = s->traj_off[t];
        uw[t] = wtot;
        wtot += s->problems[s->traj_problem[t]].m;
    }
    DevBuf d_ui, d_us, d_uw, d_w, d_hs, d_ns, d_loss, d_gx, d_gw, d_uc, d_ck;
    const size_t vb = av->bytes;
    AS_CUDA(d_ui.alloc(sizeof(int) * nt));
    AS_CUDA(d_us.alloc(sizeof(long long) * nt));
    AS_CUDA(d_uw.alloc(sizeof(long long) * nt));
    AS_CUDA(d_hs.alloc(sizeof(double) * (size_t)nt * max_steps));
    AS_CUDA(d_ns.alloc(sizeof(int) * (nt + 2)));
    AS_CUDA(d_loss.alloc(sizeof(double) * nt));
    AS_CUDA(d_gx.alloc(vb * (size_t)s->total_values));
    AS_CUDA(d_gw.alloc(sizeof(double) * (size_t)std::max<long long>(wtot, 1)));
    AS_CUDA(cudaMemcpy(d_ui.p, ui.data(), sizeof(int) * nt, cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemcpy(d_us.p, us.data(), sizeof(long long) * nt, cudaMemcpyHostToDevice));
    AS_CUDA(cudaMemcpy(d_uw.p, uw.data(), sizeof(long long) * nt, cudaMemcpyHostToDevice));
    if (weights) {
        AS_CUDA(d_w.alloc(sizeof(double) * (size_t)std::max<long long>(wtot, 1)));
        AS_CUDA(cudaMemcpy(d_w.p, weights, sizeof(double) * wtot, cudaMemcpyHostToDevice));
    }
    AS_CUDA(cudaMemset(d_ns.p, 0, sizeof(int) * (nt + 2)));

    AdjointParams P;
    P.inst = s->pool.inst.as<DevInstance>();
    P.unit_inst = d_ui.as<int>();
    P.unit_state = d_us.as<long long>();
    P.unit_wofs = d_uw.as<long long>();
    P.x0 = s->states.p;
    P.weights = weights ? d_w.as<double>() : nullptr;
    P.hs = d_hs.as<double>();
    P.nsteps = d_ns.as<int>();
    P.ckpt = nullptr;
    P.unit_ckpt = nullptr;
    P.loss = d_loss.as<double>();
    P.grad_x0 = d_gx.p;
    P.grad_w = d_gw.as<double>();
    P.num_units = nt;
    P.max_steps = max_steps;
    P.eps = s->eps;
    P.t_end = t_end;

    auto launch = [&](AdjFn fn) -> int {
        AS_CUDA(raise_smem_limit((const void*)fn, smem));
        int occ = 0;
        AS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, bt, smem));
        if (occ < 1) return fail(AS_ERR_UNSUPPORTED, "adjoint launch shape does not fit on an SM");
        void* args[] = {&P};
        AS_CUDA(cudaLaunchKernel((const void*)fn, dim3(std::min(nt, s->sm_count * occ)), dim3(bt), args, smem,
                                 s->stream));
        AS_CUDA(cudaStreamSynchronize(s->stream));
        return AS_OK;
    };
    int r = launch(av->fwd);
    if (r) return r;
    std::vector<int> ns(nt);
    AS_CUDA(cudaMemcpy(ns.data(), d_ns.p, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    std::vector<long long> uc(nt);
    long long ctot = 0;
    for (int t = 0; t < nt; t++) {
        if (ns[t] < 0)
            return fail(AS_ERR_UNSUPPORTED, ns[t] == -1 ? "adjoint: more than max_steps steps to reach t_end"
                                                        : "adjoint: step size underflow");
        uc[t] = ctot;
        ctot += (long long)ns[t] * (s->problems[s->traj_problem[t]].n + s->problems[s->traj_problem[t]].m);
    }
    AS_CUDA(d_uc.alloc(sizeof(long long) * nt));
    AS_CUDA(d_ck.alloc(vb * (size_t)std::max<long long>(ctot, 1)));
    AS_CUDA(cudaMemcpy(d_uc.p, uc.data(), sizeof(long long) * nt, cudaMemcpyHostToDevice));
    P.ckpt = d_ck.p;
    P.unit_ckpt = d_uc.as<long long>();
    r = launch(av->bwd);
    if (r) return r;
    AS_CUDA(cudaMemcpy(loss, d_loss.p, sizeof(double) * nt, cudaMemcpyDeviceToHost));
    AS_CUDA(cudaMemcpy(grad_w, d_gw.p, sizeof(double) * wtot, cudaMemcpyDeviceToHost));
    if (vb == 8) {
        AS_CUDA(cudaMemcpy(grad_x0, d_gx.p, 8 * (size_t)s->total_values, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp((size_t)s->total_values);
        AS_CUDA(cudaMemcpy(tmp.data(), d_gx.p, 4 * tmp.size(), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < tmp.size(); i++) grad_x0[i] = tmp[i];
    }
    if (nsteps) std::copy(ns.begin(), ns.end(), nsteps);
    if (step_sizes)
        AS_CUDA(cudaMemcpy(step_sizes, d_hs.p, sizeof(double) * (size_t)nt * max_steps, cudaMemcpyDeviceToHost));
    return AS_OK;
}
