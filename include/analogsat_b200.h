/*
 * analogsat_b200.h -- C ABI of the B200 (sm_100a) AnalogSAT CTDS solver.
 *
 * The reference library's boundary is a C++ template API (the AnalogSAT/solver headers):
 * SatProblem + CnfReader/CnfWriter for the CNF, ISat (the ODE right-hand side and
 * clause check), IODEInt (the RK45 integrator) and SatSolver (the run-to-solution
 * loop).  This header exports that functionality as plain `extern "C"` calls:
 * opaque handles, plain pointers and sizes, int32 status codes, no exceptions.
 * Each declaration names the reference interface it replaces (file:line, relative
 * to the reference project root).
 *
 * Conventions
 *  - Every function returns AS_OK (0) or a negative AS_ERR_* code, except the
 *    solve calls, which return AS_OK and report per-trajectory SatResult codes.
 *    as_last_error() gives the message of the last failure on the calling thread.
 *  - Public state vectors use the reference order [s_1..s_N, a_1..a_M]
 *    (AnalogSAT/solver/ISatState.h:72-127), a in linear space.
 *  - `stream` arguments are cudaStream_t values passed as void* (NULL = the
 *    legacy default stream).  Device-pointer calls are asynchronous on it.
 *  - Handles are not thread-safe; distinct handles may be used concurrently.
 *    There is no process-global device state (the reference keeps its RK45
 *    constants and buffer pointers in __constant__ symbols,
 *    AnalogSAT/cuda_sat/CudaRungeKutta.cu:42-45, so it allows one integrator
 *    per process).
 */
#ifndef ANALOGSAT_B200_H
#define ANALOGSAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------------
 * SatResult values (AnalogSAT/solver/SatResult.h:24-32), returned per trajectory. */
#define AS_SAT_SOLUTION_FOUND 0
#define AS_SAT_UNDERFLOW 1
#define AS_SAT_ODE_INTERRUPTED 2
#define AS_SAT_MAXTIME_REACHED 3
#define AS_SAT_MAXITER_REACHED 4
#define AS_SAT_UNKNOWN 5

/* call status (the reference throws: invalid_argument for bad parameters,
 * SatSolver.h:137,147,157 and CpuRungeKutta.cpp:129; runtime_error when no problem
 * is set, CpuSat.cpp:67; CudaSafe on CUDA errors, CudaUtils.cu:27-44) */
#define AS_OK 0
#define AS_ERR_BAD_INPUT (-1)
#define AS_ERR_CUDA (-2)
#define AS_ERR_NO_PROBLEM (-3)
#define AS_ERR_UNSUPPORTED (-4)
#define AS_ERR_IO (-5)
/* a device-side wait gave up (as_rhs_check): the affected outputs hold NaN */
#define AS_ERR_TIMEOUT (-6)

/* numeric modes */
#define AS_PREC_F32_LOGA 0 /* FP32 state, a_m held as log2 a_m, FP64 error norm + time */
#define AS_PREC_F64 1      /* FP64 state, linear a_m: bit-for-bit the reference RHS */

typedef struct as_problem as_problem;
typedef struct as_solver as_solver;

/* Message of the last failed call on this thread ("" if none). Returns its length. */
int32_t as_last_error(char* buf, int32_t buf_len);

/* Library / device information: number of SMs of `device`, or a negative error. */
int32_t as_device_sm_count(int32_t device);

/* ---- problems (SatProblem, AnalogSAT/problem/SatProblem.h:26-63) ----------- */

/* SatProblem::AddClauses(literals, lengths) (SatProblem.cpp:64-95): zero literals
 * are filtered, empty clauses dropped, N = max |literal|, K = max clause length. */
int32_t as_problem_create(const int32_t* literals, const int32_t* lengths, int32_t num_clauses,
                          as_problem** out);

/* CnfReader::Read (AnalogSAT/io/CnfReader.cpp:48-141); msg receives the reader's message.
 * Literals beyond +-(2^31 - 1) fail with "literal out of range". */
int32_t as_problem_read_cnf(const char* path, as_problem** out, char* msg, int32_t msg_len);
/* The same reader for very large files: the preamble is read on the host, the clause
 * body is copied once to `device` and tokenised there (every maximal run of digits is
 * one literal; the first malformed byte, sign without digits, end of file or
 * out-of-range literal before the M-th zero fails).  Results, messages and error
 * codes are those of as_problem_read_cnf. */
int32_t as_problem_read_cnf_device(const char* path, int32_t device, as_problem** out, char* msg,
                                   int32_t msg_len);

/* CnfWriter::Write (AnalogSAT/io/CnfWriter.cpp:49-74). */
int32_t as_problem_write_cnf(const as_problem* p, const char* path);

/* SatProblem::Get_N / Get_M / Get_K (SatProblem.h:58-60). */
int32_t as_problem_get_nmk(const as_problem* p, int32_t* n, int32_t* m, int32_t* k);

/* SatProblem::GetAllClauses (SatProblem.cpp:104-110): literals must hold the total
 * literal count (as_problem_num_literals), lengths M entries. */
int32_t as_problem_num_literals(const as_problem* p);
int32_t as_problem_get_clauses(const as_problem* p, int32_t* literals, int32_t* lengths);

/* Device-layout diagnostics of the packing for `precision` (no reference
 * counterpart): contribution slots, largest variable degree, shared-memory
 * wavefronts of one spin-gather pass after bank-aware clause grouping (the ideal is
 * k * ceil(M/32)), and whether the shared-memory kernels accept the instance.
 * `precision` may also be AS_LAYOUT_F32_PAIR, the packing of the FP32 device RHS
 * (as_rhs_f32) that holds two states per shared element; its wavefronts are
 * counted per 16-lane half-warp (ideal k * ceil(M/16)). */
#define AS_LAYOUT_F32_PAIR 2
int32_t as_problem_layout_stats(const as_problem* p, int32_t precision, int32_t* nslots,
                                int32_t* max_degree, int64_t* bank_wavefronts, int32_t* compact);

void as_problem_free(as_problem* p);

/* CTDS variant of a problem, the reference's choice of ISat class: AS_MODEL_CTDS is
 * CpuSat / CudaSat1-3, AS_MODEL_TANH is CpuSatTanh / CudaSatTanh1-3 with slope q
 * (AnalogSAT/cpu_sat/CpuSatTanh.h:35, Set_Q at :92; default q = 1.1,
 * CpuSatTanh.cpp:40): ds_i = sum_m knorm a_m |K_mi| tanh(q (1 - c_mi s_i)) c_mi.
 * Device RHS (as_rhs_*) and solvers created afterwards use it.  The streamed
 * solver, thread-block clusters and the adjoint support AS_MODEL_CTDS with b = 0
 * only (AS_ERR_UNSUPPORTED otherwise). */
#define AS_MODEL_CTDS 0
#define AS_MODEL_TANH 1
int32_t as_problem_set_model(as_problem* p, int32_t model, double q);
/* ISat::Set_B (AnalogSAT/solver/ISat.h:53; applied in CpuSat.cpp:229-238): adds
 * mean(a) (M/N) b knorm^2 (pi/2) sin(pi s_i) to ds_i; b >= 0, 0 = off (default). */
int32_t as_problem_set_bias(as_problem* p, double b);
int32_t as_problem_get_model(const as_problem* p, int32_t* model, double* q, double* b);

/* ---- device primitives (ISat, AnalogSAT/solver/ISat.h:31-87) -------------- */

/* ISat::GetDerivatives over `num_states` states at once (CpuSat.cpp:65-94,
 * CudaSat1.cu:501-531).  x and dxdt are DEVICE pointers to num_states public-layout
 * vectors of N+M values each (FP32).  logspace = 1: the a-block of x holds
 * u = log2 a and receives du/dt = K^2 / ln 2 (the solver's internal form). */
int32_t as_rhs_f32(as_problem* p, const float* x, float* dxdt, int32_t num_states,
                   int32_t logspace, void* stream);
/* FP64 variant, linear a: bit-identical to CpuSat<double>::GetDerivatives. */
int32_t as_rhs_f64(as_problem* p, const double* x, double* dxdt, int32_t num_states, void* stream);
/* Device-side status of the earlier asynchronous as_rhs_* calls on p (no reference
 * counterpart; the reference RHS has no waits).  The FP32 RHS moves states through
 * shared memory with asynchronous bulk copies and waits for them at most two
 * seconds; a copy that has not completed by then (a broken device, never a normal
 * run) leaves NaN in the outputs of the states that CTA had left and sets a status
 * word of the problem.  as_rhs_check waits for `stream`, reads and clears that word,
 * and returns AS_ERR_TIMEOUT if it was set, else AS_OK. */
int32_t as_rhs_check(as_problem* p, void* stream);

/* ISat::GetClauseViolationCount over many states (CpuSat.cpp:136-173,
 * CudaSat1.cu:484-498).  x: DEVICE pointer to num_states public vectors (only the
 * first N entries of each, the spins, are read); counts: DEVICE int32[num_states]. */
int32_t as_violations_f32(as_problem* p, const float* x, int32_t* counts, int32_t num_states,
                          void* stream);
int32_t as_violations_f64(as_problem* p, const double* x, int32_t* counts, int32_t num_states,
                          void* stream);

/* ---- batched solver (SatSolver<T,S>, AnalogSAT/solver/SatSolver.h:41-356) -- */

/* SatSolver(ISat, IODEInt) + SetProblem (SatSolver.h:54-71, 207-218) for a batch of
 * instances.  The solver keeps its own device copy of every problem (the handles
 * may be freed afterwards).  precision: AS_PREC_*.  device: CUDA ordinal (-1 =
 * current). */
int32_t as_solver_create(const as_problem* const* problems, int32_t num_problems,
                         int32_t precision, int32_t device, as_solver** out);
void as_solver_free(as_solver* s);

/* SatSolver setters (SatSolver.h:133-160; defaults maxTime 100, maxSteps 1e5,
 * batchSize 20 at 60-62) and CpuRungeKutta::SetEpsilon (CpuRungeKutta.cpp:126-131,
 * default 1e-4, valid range [1e-16, 1]). */
int32_t as_solver_set_max_time(as_solver* s, double max_time);
int32_t as_solver_set_max_steps(as_solver* s, int32_t max_steps);
int32_t as_solver_set_batch_size(as_solver* s, int32_t batch_size);
int32_t as_solver_set_epsilon(as_solver* s, double eps);
/* Wall-clock budget per solve call in seconds (0 = none).  Trajectories still running
 * when it expires stop with AS_SAT_ODE_INTERRUPTED -- the reference frontend gets the
 * same result from its callback returning false (Frontend/src/bench_runner.cpp:225-229). */
int32_t as_solver_set_wall_budget(as_solver* s, double seconds);
/* 1: the first trajectory that solves an instance stops that instance's other
 * trajectories (AS_SAT_ODE_INTERRUPTED).  0 (default): every trajectory runs on. */
int32_t as_solver_set_stop_on_first(as_solver* s, int32_t flag);
/* 1: keep, per trajectory, the Boolean assignment with the fewest unsat clauses
 * seen at any check (MAXSAT runs); read it with as_solver_get_best_assignment. */
int32_t as_solver_set_track_best(as_solver* s, int32_t flag);

/* SatSolver::SetSatState (SatSolver.h:183-192) for a set of trajectories.  Trajectory
 * t solves problem problem_index[t] from states + offset_t, where the host arrays are
 * concatenated public vectors (N_p + M_p values each, in trajectory order). */
int32_t as_solver_set_states_f64(as_solver* s, const int32_t* problem_index, int32_t num_traj,
                                 const double* states);
int32_t as_solver_set_states_f32(as_solver* s, const int32_t* problem_index, int32_t num_traj,
                                 const float* states);
/* Same with the states already on the device (in the solver's precision:
 * float for AS_PREC_F32_LOGA, double for AS_PREC_F64), copied device-to-device. */
int32_t as_solver_set_states_device(as_solver* s, const int32_t* problem_index, int32_t num_traj,
                                    const void* states_dev, void* stream);

/* SatSolver::SetRandomInitialState (SatSolver.h:195-201; ISat::SetRandomState,
 * CpuSat.cpp:123-133, CudaSat1.cu:452-464) for a set of trajectories, generated in
 * device memory (no host state, no host-to-device copy of it).  Uniforms u in [0, 1)
 * come from Philox4x64-10 keyed by (seed, 0): draw d is output d%4 of the block with
 * counter d/4 + 1, u = (x >> 11) * 2^-53 -- the stream of numpy's
 * Generator(Philox(key=seed)) -- and the trajectories draw from it in order.
 *   AS_IC_SPIN_UNIFORM: N draws per trajectory, s = 2u - 1, a_m = a0 (> 0); T equal
 *     trajectories get numpy's .uniform(-1, 1, (T, N)) row by row.
 *   AS_IC_REFERENCE: N + M draws, s = 2u - 1, a = u + 1 (the reference's transform,
 *     KernelSetInitial1, CudaSatBase.cu:37-55); a0 is ignored.
 * FP32 solvers store each value rounded to nearest from double. */
#define AS_IC_SPIN_UNIFORM 0
#define AS_IC_REFERENCE 1
int32_t as_solver_set_random_states(as_solver* s, const int32_t* problem_index, int32_t num_traj,
                                    uint64_t seed, int32_t distribution, double a0);

/* SatSolver::Solve (SatSolver.h:162-165, DoSolve 273-355) for every trajectory, in
 * one persistent launch.  Blocks until done.  Per-trajectory results via
 * as_solver_get_results. */
int32_t as_solver_solve(as_solver* s);
/* Asynchronous form: enqueue on `stream`; completion via as_solver_sync. */
int32_t as_solver_solve_async(as_solver* s, void* stream);
int32_t as_solver_sync(as_solver* s);

/* Per-trajectory statistics (SatSolver getters, SatSolver.h:77-130): any pointer may
 * be NULL.  status: SatResult code; time: GetElapsedTime; steps: GetStepCount; rhs:
 * GetRhsCount; attempts: IODEInt::GetAttemptCount; violations:
 * GetLastClauseViolationCount; min_violations: smallest count seen; last_step:
 * GetLastStepSize. */
int32_t as_solver_get_results(as_solver* s, int32_t* status, double* time, int32_t* steps,
                              int32_t* rhs, int32_t* attempts, int32_t* violations,
                              int32_t* min_violations, double* last_step);

/* SatSolver::GetSatState().CopyTo (SatSolver.h:168-169): final public states of all
 * trajectories, concatenated as in as_solver_set_states_*. */
int32_t as_solver_get_states_f64(as_solver* s, double* states);
int32_t as_solver_get_states_f32(as_solver* s, float* states);
/* The same for one trajectory: its N + M public values, one device-to-host copy. */
int32_t as_solver_get_state_f64(as_solver* s, int32_t traj, double* state);
int32_t as_solver_get_state_f32(as_solver* s, int32_t traj, float* state);
/* Device pointer of the solver's state buffer (solver precision), for zero-copy reads. */
const void* as_solver_states_device(as_solver* s);

/* Best assignment of trajectory t (needs as_solver_set_track_best(s, 1) before the
 * solve): bits[w] bit b = variable 32w+b+1 TRUE.  bits holds ceil(N/32) words. */
int32_t as_solver_get_best_assignment(as_solver* s, int32_t traj, uint32_t* bits);

/* GetSatResultMessage (AnalogSAT/solver/SatResult.cpp:23-34) for a SatResult code. */
const char* as_result_message(int32_t result);
/* The reference frontend's result file for one trajectory (Frontend/src/cnf_runner.cpp:
 * 280-304): "SAT" or "INDET", then the final assignment as signed variable numbers
 * ending in 0, MiniSat-compatible.  Overwrites path. */
int32_t as_solver_write_result(as_solver* s, int32_t traj, const char* path);
/* Appends the reference bench's perf line for one trajectory (Frontend/src/
 * bench_runner.cpp:331-343): sample, GPU name, solver name, result message, wall and
 * CPU seconds of the last as_solver_solve call (the whole batched call), RHS count;
 * tab-separated. */
int32_t as_solver_append_perf(as_solver* s, int32_t traj, const char* path, const char* sample,
                              const char* solver_name);

/* Launch shape of the last solve's final launch group: threads per CTA, CTAs
 * launched, dynamic shared memory per CTA and resident CTAs per SM. */
int32_t as_solver_get_launch_shape(as_solver* s, int32_t* threads, int32_t* ctas, int32_t* smem_bytes,
                                   int32_t* ctas_per_sm);
/* Force the CTA size (a multiple of 32 in [32, 1024]) of the next solves; 0 restores
 * the automatic choice (the fewest threads that give every thread about the same
 * clause count, at least four).  Used by the autotuner. */
int32_t as_solver_force_threads(as_solver* s, int32_t threads);
/* Solver kernel of the shared-memory mode (no reference counterpart).  AS_KERNEL_AUTO
 * (default) runs FP32 instances with the plain CTDS right-hand side (no tanh variant,
 * no bias term), clause length 3 or 4 and N < 4096 on the lean kernel, whose literal
 * words carry shared-memory byte offsets and whose RK vectors are interleaved per
 * element: the same integrator and arithmetic with fewer instructions per clause.
 * AS_KERNEL_GENERIC keeps every instance on the general kernel.  Results of the two
 * agree to FP32 rounding. */
#define AS_KERNEL_AUTO 0
#define AS_KERNEL_GENERIC 1
int32_t as_solver_set_kernel(as_solver* s, int32_t kernel);
/* Name of the solver kernel of the last solve's final launch group ("" before the
 * first solve; no reference counterpart). */
const char* as_solver_kernel_name(const as_solver* s);
/* Where a trajectory lives while it is integrated (no reference counterpart):
 * AS_STORAGE_AUTO picks the streamed solver when every instance has N + M >= 2^19
 * state elements, else shared memory when the instance fits one SM, else global
 * storage (a per-CTA slab in device memory); the others force one.
 * AS_STORAGE_STREAM: trajectories of an instance are grouped by eight with their
 * states interleaved in device memory, and every RK attempt runs as per-stage
 * kernels over the whole GPU, replayed from a CUDA graph; each trajectory keeps its
 * own step size and the reference's counters.  It is host driven: a solve returns
 * when the run is over (as_solver_solve_async first waits for the caller's stream).
 * Solves fail with AS_ERR_UNSUPPORTED when a forced mode cannot hold an instance. */
#define AS_STORAGE_AUTO 0
#define AS_STORAGE_SHARED 1
#define AS_STORAGE_GLOBAL 2
#define AS_STORAGE_STREAM 3
int32_t as_solver_set_storage_mode(as_solver* s, int32_t mode);
/* Clause parts per RK stage in AS_STORAGE_STREAM (no reference counterpart): the
 * clauses of an instance whose internal order is the public one (the wide packing)
 * are split into this many ranges, each range's contributions summed right after it
 * is computed (while still in L2), the row sums continuing from range to range in
 * public clause order.  0 (default) and 1: one range; up to 8.  Results do not depend
 * on it. */
int32_t as_solver_set_stream_parts(as_solver* s, int32_t parts);
/* CTAs per trajectory in global-storage mode (no reference counterpart): 0 picks
 * automatically (a thread-block cluster of 4 or 8 CTAs when there are few
 * trajectories, so that they still cover the whole GPU), 1, 4 or 8 force it. */
int32_t as_solver_set_cluster_size(as_solver* s, int32_t ctas);

/* ---- gradients (no counterpart in the reference: it has no differentiation) --
 * Weighted CTDS: a_m -> w_m a_m in the potential and the spin equation
 * (ds_i = sum_m 2 w_m a_m c_mi K_mi K_m, da_m = a_m K_m^2; w = 1 is the reference
 * ODE) and L = V(x(T)) = sum_m w_m a_m(T) K_m(s(T))^2.  For every trajectory set with
 * as_solver_set_states_* (the state buffer's current contents are x(0), a linear), the
 * adaptive RK45 controller runs to t_end (last step clamped), its accepted step sizes
 * are frozen, and the discrete adjoint of that fixed-step map gives dL/dx(0) and
 * dL/dw.  weights: NULL (all 1) or, per trajectory, M_p values in public clause order,
 * concatenated; grad_w has the same shape; grad_x0 the shape of the states (FP64);
 * loss and nsteps one value per trajectory; step_sizes (may be NULL) receives the
 * frozen step sizes, max_steps slots per trajectory.  FP32 solvers compute in FP32
 * with linear a, FP64 solvers in FP64.  Instances must fit one SM's shared memory;
 * AS_ERR_UNSUPPORTED if a trajectory needs more than max_steps steps. */
int32_t as_solver_adjoint(as_solver* s, double t_end, int32_t max_steps, const double* weights, double* loss,
                          double* grad_x0, double* grad_w, int32_t* nsteps, double* step_sizes);

/* ---- allocation-free solve (no counterpart in the reference) --------------
 * For callers that cannot allocate device memory while they run: an application
 * that has already reserved the GPU's memory for its own pool, or a fixed-latency
 * loop where a cudaMalloc (which may synchronise the device) is not allowed.
 * as_solver_solve_noalloc runs the same persistent solve kernel as
 * as_solver_solve, but keeps its per-call scratch (work counter, first-solution
 * flag, wall-clock deadline, trajectory tables) in a static device array inside the
 * library instead of in buffers owned by the solver handle, and calls no allocation
 * routine.  The array is AS_NOALLOC_SCRATCH_BYTES on every GPU that loads the
 * library, held until the process exits.
 *
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress); make that first call before any stream capture.
 *  - All calls share the array and each call re-initialises it: calls whose work
 *    overlaps on the GPU (other streams, other host threads) race.  Serialise them.
 *  - All num_traj trajectories solve problem `problem_index` of the solver (which
 *    must be < AS_NOALLOC_MAX_PROBLEM_INDEX); num_traj <= AS_NOALLOC_MAX_TRAJ,
 *    larger requests fail with AS_ERR_UNSUPPORTED.
 *  - states: DEVICE array of num_traj public states (N+M values each, float for
 *    AS_PREC_F32_LOGA solvers, double for AS_PREC_F64), initial states in, final
 *    states out.  results: DEVICE array of num_traj as_unit_result.
 *  - Only instances whose whole trajectory fits one SM's shared memory are accepted
 *    (N=1000/M=4250 in FP32 does): the global-storage and streamed modes need
 *    device buffers, so as_solver_set_storage_mode is not consulted and a larger
 *    instance fails with AS_ERR_UNSUPPORTED.  The CTA size is the one
 *    as_solver_solve picks for the same instance (or as_solver_force_threads').
 *  - The solver's settings apply (epsilon, max time/steps, batch size, wall budget,
 *    stop-on-first); best-assignment tracking is not available here.
 *  - Asynchronous on `stream`; results are valid once the stream reaches this point. */
#define AS_NOALLOC_MAX_TRAJ 65536
#define AS_NOALLOC_MAX_PROBLEM_INDEX 4096
#define AS_NOALLOC_SCRATCH_BYTES (256 + 4 * 4096 + 12 * 65536)

typedef struct as_unit_result {
    double time;            /* integrated analog time */
    double last_step;       /* last accepted step size */
    int32_t status;         /* SatResult code */
    int32_t steps;          /* accepted steps */
    int32_t attempts;       /* attempted steps */
    int32_t rhs;            /* RHS evaluations */
    int32_t violations;     /* unsat clauses at the last check */
    int32_t min_violations; /* fewest unsat clauses seen at any check */
    int32_t reserved0, reserved1;
} as_unit_result;

int32_t as_solver_solve_noalloc(as_solver* s, int32_t problem_index, int32_t num_traj, void* states,
                                as_unit_result* results, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ANALOGSAT_B200_H */
