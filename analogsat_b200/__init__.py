"""analogsat_b200 -- B200-native (sm_100a) AnalogSAT CTDS SAT/MAXSAT solver.

Python mirror of the reference library's problem/solver API over the C ABI in
``include/analogsat_b200.h`` (the C++ mirror is ``include/analogsat_b200.hpp``):

* :class:`SatProblem`  -- ``analogsat::SatProblem`` (+ ``CnfReader``/``CnfWriter``);
* :class:`SatSolver`   -- ``analogsat::SatSolver`` for a batch of instances x
  trajectories, run in one persistent CUDA launch;
* :func:`get_derivatives` / :func:`clause_violation_counts` -- ``ISat``'s
  ``GetDerivatives`` / ``GetClauseViolationCount`` over many device-resident states.

Method names follow the reference (``SetMaxTime``, ``SetSatState``, ``Solve``,
``GetStepCount`` ...); errors raise :class:`AnalogSatError`, the reference's
exceptions' counterpart.  Every call goes to the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from enum import IntEnum

import numpy as np

from . import _abi
from ._abi import AnalogSatError, AS_PREC_F32_LOGA, AS_PREC_F64, check, load

__all__ = [
    "SatResult", "SatProblem", "SatSolver", "AnalogSatError", "AS_PREC_F32_LOGA", "AS_PREC_F64",
    "get_derivatives", "rhs_check", "clause_violation_counts", "load", "sat_result_message",
]


class SatResult(IntEnum):
    """AnalogSAT/solver/SatResult.h:24-32"""
    SAT_SOLUTION_FOUND = 0
    SAT_UNDERFLOW = 1
    SAT_ODE_INTERRUPTED = 2
    SAT_MAXTIME_REACHED = 3
    SAT_MAXITER_REACHED = 4
    SAT_UNKNOWN = 5


_MESSAGES = {0: "solution found", 1: "underflow", 2: "user interrupt", 3: "maximum time reached",
             4: "maximum steps reached"}


def sat_result_message(r: int) -> str:
    """GetSatResultMessage (AnalogSAT/solver/SatResult.cpp:21-33)."""
    return _MESSAGES.get(int(r), "unknown result")


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a: np.ndarray, t=C.c_int32):
    return a.ctypes.data_as(C.POINTER(t))


class SatProblem:
    """A CNF formula (AnalogSAT/problem/SatProblem.h:26-63)."""

    def __init__(self, handle=None):
        self._lib = load()
        self._h = handle

    @classmethod
    def from_arrays(cls, literals, lengths) -> "SatProblem":
        """SatProblem::AddClauses(literals, lengths) (SatProblem.cpp:64-95)."""
        lits, lens = _i32(literals), _i32(lengths)
        if lens.size and lens.sum() != lits.size:
            raise AnalogSatError(_abi.AS_ERR_BAD_INPUT, "lengths do not sum to the literal count")
        h = C.c_void_p()
        check(load().as_problem_create(_ptr(lits), _ptr(lens), int(lens.size), C.byref(h)))
        return cls(h)

    @classmethod
    def from_clauses(cls, clauses) -> "SatProblem":
        """SatProblem::AddClauses(vector<vector<int>>) (SatProblem.cpp:97-103)."""
        lens = [len(c) for c in clauses]
        lits = [l for c in clauses for l in c]
        return cls.from_arrays(lits, lens)

    @classmethod
    def read_cnf(cls, path: str, device: int | None = None) -> "SatProblem":
        """CnfReader::Read (AnalogSAT/io/CnfReader.cpp:48-141).  With `device`, the
        clause body is tokenised on that GPU (same results and messages)."""
        h = C.c_void_p()
        msg = C.create_string_buffer(256)
        if device is None:
            check(load().as_problem_read_cnf(path.encode(), C.byref(h), msg, 256))
        else:
            check(load().as_problem_read_cnf_device(path.encode(), int(device), C.byref(h), msg, 256))
        p = cls(h)
        p.message = msg.value.decode()
        return p

    def write_cnf(self, path: str) -> None:
        """CnfWriter::Write (AnalogSAT/io/CnfWriter.cpp:49-74)."""
        check(self._lib.as_problem_write_cnf(self._h, path.encode()))

    def _nmk(self):
        n, m, k = C.c_int32(), C.c_int32(), C.c_int32()
        check(self._lib.as_problem_get_nmk(self._h, C.byref(n), C.byref(m), C.byref(k)))
        return n.value, m.value, k.value

    def Get_N(self) -> int:
        return self._nmk()[0]

    def Get_M(self) -> int:
        return self._nmk()[1]

    def Get_K(self) -> int:
        return self._nmk()[2]

    @property
    def n(self) -> int:
        return self.Get_N()

    @property
    def m(self) -> int:
        return self.Get_M()

    @property
    def k(self) -> int:
        return self.Get_K()

    def GetAllClauses(self):
        """SatProblem::GetAllClauses (SatProblem.cpp:104-110) -> (literals, lengths)."""
        nl = check(self._lib.as_problem_num_literals(self._h))
        lits = np.zeros(max(nl, 1), np.int32)
        lens = np.zeros(max(self.m, 1), np.int32)
        check(self._lib.as_problem_get_clauses(self._h, _ptr(lits), _ptr(lens)))
        return lits[:nl], lens[: self.m]

    def set_model(self, tanh: bool = False, q: float = 1.1):
        """The reference's choice of CTDS class: CpuSat (tanh=False) or CpuSatTanh with
        slope q (Set_Q).  Device RHS calls and solvers created afterwards use it."""
        check(self._lib.as_problem_set_model(self._h, _abi.AS_MODEL_TANH if tanh else _abi.AS_MODEL_CTDS,
                                             float(q)))
        return self

    def set_bias(self, b: float):
        """ISat::Set_B: the bias term mean(a) (M/N) b knorm^2 (pi/2) sin(pi s_i); 0 = off."""
        check(self._lib.as_problem_set_bias(self._h, float(b)))
        return self

    def Set_B(self, b: float):
        return self.set_bias(b)

    def model(self) -> dict:
        t, q, b = C.c_int32(), C.c_double(), C.c_double()
        check(self._lib.as_problem_get_model(self._h, C.byref(t), C.byref(q), C.byref(b)))
        return dict(tanh=t.value == _abi.AS_MODEL_TANH, q=q.value, b=b.value)

    def layout_stats(self, precision: int = AS_PREC_F32_LOGA) -> dict:
        a, b, d = C.c_int32(), C.c_int32(), C.c_int32()
        c = C.c_int64()
        check(self._lib.as_problem_layout_stats(self._h, precision, C.byref(a), C.byref(b),
                                                C.byref(c), C.byref(d)))
        return dict(nslots=a.value, max_degree=b.value, bank_wavefronts=c.value,
                    compact=bool(d.value))

    def __del__(self):
        try:
            if self._h:
                self._lib.as_problem_free(self._h)
        except Exception:
            pass


def _stream_ptr(stream):
    """A CUDA stream handle: an int (cudaStream_t), an object with .cuda_stream (a
    torch.cuda.Stream), or None for torch's current stream."""
    if stream is None:
        try:
            import torch
            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:
            return C.c_void_p(0)
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


def get_derivatives(problem: SatProblem, x, out=None, logspace: bool = False, stream=None):
    """ISat::GetDerivatives for a [B, N+M] CUDA tensor of public states (float32 or
    float64).  float64 follows CpuSat<double> bit for bit; float32 with logspace=True
    treats the a-block as log2 a and returns d(log2 a)/dt = K^2 / ln 2."""
    import torch
    if not x.is_cuda:
        raise AnalogSatError(_abi.AS_ERR_BAD_INPUT, "get_derivatives needs a CUDA tensor")
    x = x.contiguous()
    if out is None:
        out = torch.empty_like(x)
    B = x.shape[0] if x.dim() == 2 else 1
    lib = load()
    if x.dtype == torch.float64:
        if logspace:
            raise AnalogSatError(_abi.AS_ERR_UNSUPPORTED, "log-space RHS is FP32 only")
        check(lib.as_rhs_f64(problem._h, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), B,
                             _stream_ptr(stream)))
    elif x.dtype == torch.float32:
        check(lib.as_rhs_f32(problem._h, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), B,
                             int(logspace), _stream_ptr(stream)))
    else:
        raise AnalogSatError(_abi.AS_ERR_BAD_INPUT, "x must be float32 or float64")
    return out


def rhs_check(problem: SatProblem, stream=None) -> None:
    """Waits for `stream` and raises AnalogSatError(AS_ERR_TIMEOUT) if a device RHS on
    `problem` gave up waiting for one of its bulk copies (its outputs then hold NaN)."""
    check(load().as_rhs_check(problem._h, _stream_ptr(stream)))


def clause_violation_counts(problem: SatProblem, x, stream=None):
    """ISat::GetClauseViolationCount for a [B, N+M] CUDA tensor -> int32[B] (device)."""
    import torch
    x = x.contiguous()
    B = x.shape[0] if x.dim() == 2 else 1
    out = torch.empty(B, dtype=torch.int32, device=x.device)
    lib = load()
    fn = lib.as_violations_f64 if x.dtype == torch.float64 else lib.as_violations_f32
    check(fn(problem._h, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), B,
             _stream_ptr(stream)))
    return out


class SatSolver:
    """Batched counterpart of ``SatSolver<TFloat,TState>`` (AnalogSAT/solver/SatSolver.h).

    One solver holds several instances; ``SetSatStates`` assigns trajectories
    (instance index + initial public state each) and ``Solve`` runs all of them to
    their SatResult in one persistent launch.  Defaults are the reference's:
    maxTime 100, maxSteps 1e5, batch 20, eps 1e-4.
    """

    def __init__(self, problems, precision: int = AS_PREC_F32_LOGA, device: int = -1):
        if isinstance(problems, SatProblem):
            problems = [problems]
        self._lib = load()
        self.problems = list(problems)
        self.precision = precision
        arr = (C.c_void_p * len(self.problems))(*[p._h for p in self.problems])
        h = C.c_void_p()
        check(self._lib.as_solver_create(arr, len(self.problems), precision, device, C.byref(h)))
        self._h = h
        self._nm = [(p.n, p.m) for p in self.problems]
        self._traj_problem = None

    # -- configuration (SatSolver.h:133-160, CpuRungeKutta.cpp:126-131) --
    def SetMaxTime(self, v: float):
        check(self._lib.as_solver_set_max_time(self._h, float(v)))

    def SetMaxSteps(self, v: int):
        check(self._lib.as_solver_set_max_steps(self._h, int(v)))

    def SetBatchSize(self, v: int):
        check(self._lib.as_solver_set_batch_size(self._h, int(v)))

    def SetEpsilon(self, v: float):
        check(self._lib.as_solver_set_epsilon(self._h, float(v)))

    def SetWallBudget(self, seconds: float):
        check(self._lib.as_solver_set_wall_budget(self._h, float(seconds)))

    def SetStopOnFirst(self, flag: bool):
        check(self._lib.as_solver_set_stop_on_first(self._h, int(bool(flag))))

    def SetTrackBest(self, flag: bool):
        check(self._lib.as_solver_set_track_best(self._h, int(bool(flag))))

    def ForceThreads(self, threads: int):
        check(self._lib.as_solver_force_threads(self._h, int(threads)))

    def SetKernel(self, kernel: int):
        """Shared-memory solver kernel: _abi.AS_KERNEL_AUTO (the lean FP32 kernel where the
        instance qualifies) or _abi.AS_KERNEL_GENERIC."""
        check(self._lib.as_solver_set_kernel(self._h, int(kernel)))

    def SetClusterSize(self, ctas: int):
        """CTAs per trajectory in global-storage mode: 0 automatic, 1, 4 or 8."""
        check(self._lib.as_solver_set_cluster_size(self._h, int(ctas)))

    def SetStreamParts(self, parts: int):
        """Clause parts per RK stage of the streamed solver (0: from the L2 budget)."""
        check(self._lib.as_solver_set_stream_parts(self._h, int(parts)))

    def SetStorageMode(self, mode: int):
        """0 automatic, 1 shared memory only, 2 global storage (per-CTA slab) only,
        3 streamed (eight trajectories per lane group, per-stage kernels over the GPU)."""
        check(self._lib.as_solver_set_storage_mode(self._h, int(mode)))

    # -- states (SatSolver::SetSatState, SatSolver.h:183-192) --
    def SetSatStates(self, problem_index, states, stream=None):
        """states: host array of the concatenated public vectors, or a CUDA tensor
        (copied device-to-device on `stream` -- a cudaStream_t handle or a
        torch.cuda.Stream -- default the current torch stream)."""
        pi = _i32(problem_index)
        self._traj_problem = pi.copy()
        try:
            import torch
            is_tensor = isinstance(states, torch.Tensor)
        except ImportError:
            is_tensor = False
        if is_tensor and states.is_cuda:
            check(self._lib.as_solver_set_states_device(
                self._h, _ptr(pi), int(pi.size), C.c_void_p(states.data_ptr()),
                _stream_ptr(stream)))
            return
        if is_tensor:
            states = states.numpy()
        st = np.ascontiguousarray(states)
        if st.dtype == np.float32:
            check(self._lib.as_solver_set_states_f32(self._h, _ptr(pi), int(pi.size),
                                                     st.ctypes.data_as(C.c_void_p)))
        else:
            st = np.ascontiguousarray(st, np.float64)
            check(self._lib.as_solver_set_states_f64(self._h, _ptr(pi), int(pi.size),
                                                     st.ctypes.data_as(C.c_void_p)))

    IC_DISTRIBUTIONS = {"spin_uniform": 0, "reference": 1}

    def SetRandomInitialState(self, problem_index, seed: int, distribution: str = "spin_uniform",
                              a0: float = 1.0):
        """SatSolver::SetRandomInitialState (SatSolver.h:195-201) for a set of
        trajectories, generated on the device from Philox4x64-10 keyed by seed.
        "spin_uniform": s ~ U(-1, 1), a = a0 -- for T trajectories of one problem the
        states equal instances.initial_states(N, M, T, seed, a0);  "reference": the
        reference's ISat::SetRandomState transform, s = 2u - 1, a = u + 1."""
        pi = _i32(problem_index)
        self._traj_problem = pi.copy()
        check(self._lib.as_solver_set_random_states(self._h, _ptr(pi), int(pi.size), int(seed),
                                                    self.IC_DISTRIBUTIONS[distribution], float(a0)))

    def SetSatState(self, state, problem: int = 0):
        """Single-trajectory form of SatSolver::SetSatState(vector)."""
        self.SetSatStates([problem], np.asarray(state))

    def Solve(self):
        """SatSolver::Solve for every trajectory; returns the SatResult array."""
        check(self._lib.as_solver_solve(self._h))
        return self.results()["status"]

    def SolveAsync(self, stream=None):
        """Enqueue the solve without waiting (as_solver_solve_async): on the solver's own
        stream, or on `stream` (a cudaStream_t handle or a torch.cuda.Stream), ordered
        after the states set before and before the reads queued after; Sync() waits."""
        check(self._lib.as_solver_solve_async(self._h, _stream_ptr(stream) if stream else None))

    def Sync(self):
        check(self._lib.as_solver_sync(self._h))

    def results(self) -> dict:
        n = len(self._traj_problem)
        st = np.zeros(n, np.int32); tm = np.zeros(n); sp = np.zeros(n, np.int32)
        rh = np.zeros(n, np.int32); at = np.zeros(n, np.int32); vi = np.zeros(n, np.int32)
        mv = np.zeros(n, np.int32); hd = np.zeros(n)
        check(self._lib.as_solver_get_results(
            self._h, _ptr(st), _ptr(tm, C.c_double), _ptr(sp), _ptr(rh), _ptr(at), _ptr(vi),
            _ptr(mv), _ptr(hd, C.c_double)))
        return dict(status=st, time=tm, steps=sp, rhs=rh, attempts=at, violations=vi,
                    min_violations=mv, last_step=hd)

    def GetSatStates(self, dtype=np.float64, out=None) -> np.ndarray:
        """Final public states, concatenated (SatSolver::GetSatState().CopyTo).
        `out` may be a preallocated (e.g. pinned) host array of the right size/dtype."""
        total = int(sum(sum(self._nm[p]) for p in self._traj_problem))
        if out is None:
            out = np.zeros(total, dtype)
        dtype = out.dtype
        if out.size != total or not out.flags.c_contiguous:
            raise AnalogSatError(_abi.AS_ERR_BAD_INPUT, "out has the wrong size or layout")
        fn = (self._lib.as_solver_get_states_f32 if dtype == np.float32
              else self._lib.as_solver_get_states_f64)
        check(fn(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def WriteResult(self, traj: int, path: str):
        """The reference frontend's MiniSat-compatible result file (SAT / INDET + assignment)."""
        check(self._lib.as_solver_write_result(self._h, int(traj), os.fsencode(path)))

    def AppendPerf(self, traj: int, path: str, sample: str, solver_name: str = "analogsat_b200"):
        """Appends the reference bench's tab-separated perf line for one trajectory."""
        check(self._lib.as_solver_append_perf(self._h, int(traj), os.fsencode(path), sample.encode(),
                                              solver_name.encode()))

    def GetSatState(self, traj: int = 0, dtype=np.float64) -> np.ndarray:
        """Final public state of one trajectory (one device-to-host copy)."""
        if not 0 <= traj < len(self._traj_problem):
            raise AnalogSatError(_abi.AS_ERR_BAD_INPUT, "trajectory index out of range")
        n, m = self._nm[self._traj_problem[traj]]
        out = np.zeros(n + m, dtype)
        fn = (self._lib.as_solver_get_state_f32 if out.dtype == np.float32
              else self._lib.as_solver_get_state_f64)
        check(fn(self._h, int(traj), out.ctypes.data_as(C.c_void_p)))
        return out

    def GetBestAssignment(self, traj: int) -> np.ndarray:
        n, _ = self._nm[self._traj_problem[traj]]
        bits = np.zeros((n + 31) // 32, np.uint32)
        check(self._lib.as_solver_get_best_assignment(self._h, int(traj),
                                                      bits.ctypes.data_as(C.c_void_p)))
        return ((bits[np.arange(n) // 32] >> (np.arange(n) % 32).astype(np.uint32)) & 1).astype(bool)

    def Adjoint(self, t_end: float, weights=None, max_steps: int = 4096) -> dict:
        """Gradients of L = sum_m w_m a_m(T) K_m(T)^2 w.r.t. x(0) and w for every
        trajectory (see as_solver_adjoint); x(0) is the current state buffer."""
        nt = len(self._traj_problem)
        ms = [self._nm[p][1] for p in self._traj_problem]
        total = int(sum(sum(self._nm[p]) for p in self._traj_problem))
        loss = np.zeros(nt); gx = np.zeros(total); gw = np.zeros(max(sum(ms), 1))
        ns = np.zeros(nt, np.int32)
        hs = np.zeros((nt, max_steps))
        wp = None
        if weights is not None:
            weights = np.ascontiguousarray(weights, np.float64)
            if weights.size != sum(ms):
                raise AnalogSatError(_abi.AS_ERR_BAD_INPUT, "weights: M values per trajectory")
            wp = weights.ctypes.data_as(C.c_void_p)
        check(self._lib.as_solver_adjoint(self._h, float(t_end), int(max_steps), wp,
                                          loss.ctypes.data_as(C.c_void_p), gx.ctypes.data_as(C.c_void_p),
                                          gw.ctypes.data_as(C.c_void_p), ns.ctypes.data_as(C.c_void_p),
                                          hs.ctypes.data_as(C.c_void_p)))
        return dict(loss=loss, grad_x0=gx, grad_w=gw[: sum(ms)], nsteps=ns,
                    step_sizes=[hs[t, : ns[t]].copy() for t in range(nt)])

    def kernel_name(self) -> str:
        """Solver kernel of the last solve's final launch group."""
        return self._lib.as_solver_kernel_name(self._h).decode()

    def launch_shape(self) -> dict:
        a, b, c, d = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        check(self._lib.as_solver_get_launch_shape(self._h, C.byref(a), C.byref(b), C.byref(c),
                                                   C.byref(d)))
        return dict(threads=a.value, ctas=b.value, smem_bytes=c.value, ctas_per_sm=d.value)

    def states_device_ptr(self) -> int:
        return int(self._lib.as_solver_states_device(self._h) or 0)

    # single-trajectory getters (SatSolver.h:77-130) for trajectory 0
    def GetStepCount(self, traj: int = 0) -> int:
        return int(self.results()["steps"][traj])

    def GetRhsCount(self, traj: int = 0) -> int:
        return int(self.results()["rhs"][traj])

    def GetElapsedTime(self, traj: int = 0) -> float:
        return float(self.results()["time"][traj])

    def GetLastStepSize(self, traj: int = 0) -> float:
        return float(self.results()["last_step"][traj])

    def GetLastClauseViolationCount(self, traj: int = 0) -> int:
        return int(self.results()["violations"][traj])

    def __del__(self):
        try:
            if self._h:
                self._lib.as_solver_free(self._h)
        except Exception:
            pass
