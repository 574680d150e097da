"""TEST INFRASTRUCTURE ONLY -- not part of the product.

ctypes bindings for the two CPU checkers built by ``oracle/Makefile``:

* ``Oracle``    -- ``liboracle.so``, our FP64 C restatement of the CTDS path
  (``oracle/ctds_oracle.c``);
* ``Reference`` -- ``_ref/libanalogsat_ref.so``, the reference AnalogSAT CPU solver
  and MiniSat compiled from the reference's own sources plus ``ref_shim.cpp``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm import this module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libanalogsat_ref.so")
REFCUDA_SO = os.path.join(HERE, "_ref", "libanalogsat_refcuda.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


REFERENCE_ROOT = os.environ.get("ANALOGSAT_REF", "/root/reference")


def build(reference_root: str | None = REFERENCE_ROOT) -> None:
    """Compile the C restatement, and the reference solver when its sources exist
    (the reference source tree comes from $ANALOGSAT_REF, default /root/reference)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if reference_root and os.path.isdir(reference_root):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "refcuda", f"REF={reference_root}"], check=True)


def _flat(clauses):
    lens = np.array([len(c) for c in clauses], dtype=np.int32)
    lits = np.array([l for c in clauses for l in c], dtype=np.int32)
    return lits, lens


class Oracle:
    """FP64 C restatement (checker)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(None)
        L = C.CDLL(path)
        L.orc_problem_new.restype = C.c_void_p
        L.orc_problem_new.argtypes = [_i32p, _i32p, C.c_int]
        L.orc_problem_free.argtypes = [C.c_void_p]
        L.orc_problem_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3
        L.orc_rhs.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int]
        L.orc_violations.restype = C.c_int
        L.orc_violations.argtypes = [C.c_void_p, _f64p]
        L.orc_steps.restype = C.c_int
        L.orc_steps.argtypes = [C.c_void_p, _f64p, C.c_double, C.c_int, C.c_int, _f64p, _f64p,
                                _i32p, _i32p, _f64p]
        L.orc_solve.restype = C.c_int
        L.orc_solve.argtypes = [C.c_void_p, _f64p, C.c_double, C.c_double, C.c_int, C.c_int,
                                C.c_int, _f64p, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_integrate_to.restype = C.c_int
        L.orc_integrate_to.argtypes = [C.c_void_p, _f64p, C.c_double, C.c_double, C.c_int, C.c_int,
                                       _f64p, C.POINTER(C.c_double)]
        L.orc_potential.restype = C.c_double
        L.orc_potential.argtypes = [C.c_void_p, _f64p, C.c_void_p]
        L.orc_record_steps.restype = C.c_int
        L.orc_record_steps.argtypes = [C.c_void_p, _f64p, C.c_double, C.c_double, C.c_int, _f64p]
        L.orc_fixed_loss.restype = C.c_double
        L.orc_fixed_loss.argtypes = [C.c_void_p, _f64p, C.c_void_p, _f64p, C.c_int, C.c_void_p]
        L.orc_adjoint.restype = C.c_double
        L.orc_adjoint.argtypes = [C.c_void_p, _f64p, C.c_void_p, _f64p, C.c_int, _f64p, _f64p]
        L.orc_problem_set_model.restype = None
        L.orc_problem_set_model.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        self.L = L

    class Problem:
        def __init__(self, L, lits, lens):
            self.L = L
            self.h = L.orc_problem_new(np.ascontiguousarray(lits, np.int32),
                                       np.ascontiguousarray(lens, np.int32), len(lens))
            n, m, k = C.c_int(), C.c_int(), C.c_int()
            L.orc_problem_info(self.h, C.byref(n), C.byref(m), C.byref(k))
            self.n, self.m, self.k = n.value, m.value, k.value

        def __del__(self):
            try:
                self.L.orc_problem_free(self.h)
            except Exception:
                pass

    def problem(self, lits, lens):
        return Oracle.Problem(self.L, lits, lens)

    def set_model(self, p, tanh=False, q=1.1, b=0.0):
        """CTDS variant of problem p: tanh restates CpuSatTanh (slope q); b the bias."""
        self.L.orc_problem_set_model(p.h, int(tanh), float(q), float(b))

    def problem_from_clauses(self, clauses):
        return self.problem(*_flat(clauses))

    def rhs(self, p, x, logspace=False):
        x = np.ascontiguousarray(x, np.float64)
        d = np.zeros(p.n + p.m, np.float64)
        self.L.orc_rhs(p.h, x, d, int(logspace))
        return d

    def violations(self, p, spins):
        return self.L.orc_violations(p.h, np.ascontiguousarray(spins[: p.n], np.float64))

    def steps(self, p, ic, eps, nsteps, logspace=False):
        nm = p.n + p.m
        t = np.zeros(nsteps); h = np.zeros(nsteps)
        r = np.zeros(nsteps, np.int32); a = np.zeros(nsteps, np.int32)
        st = np.zeros(nsteps * nm)
        done = self.L.orc_steps(p.h, np.ascontiguousarray(ic, np.float64), eps, nsteps,
                                int(logspace), t, h, r, a, st)
        return dict(n=done, time=t[:done], h=h[:done], rhs=r[:done], attempts=a[:done],
                    states=st.reshape(nsteps, nm)[:done])

    def solve(self, p, ic, eps=1e-6, tmax=1e8, maxsteps=50_000_000, batch=50, logspace=False):
        fin = np.zeros(p.n + p.m)
        t = C.c_double(); st = C.c_int(); r = C.c_int(); a = C.c_int(); v = C.c_int()
        res = self.L.orc_solve(p.h, np.ascontiguousarray(ic, np.float64), eps, tmax, maxsteps,
                               batch, int(logspace), fin, C.byref(t), C.byref(st), C.byref(r),
                               C.byref(a), C.byref(v))
        return dict(result=res, state=fin, time=t.value, steps=st.value, rhs=r.value,
                    attempts=a.value, violations=v.value)

    def integrate_to(self, p, ic, t_end, eps=1e-10, logspace=False, maxsteps=10_000_000):
        out = np.zeros(p.n + p.m)
        t = C.c_double()
        steps = self.L.orc_integrate_to(p.h, np.ascontiguousarray(ic, np.float64), eps, t_end,
                                        int(logspace), maxsteps, out, C.byref(t))
        return dict(state=out, time=t.value, steps=steps)

    def record_steps(self, p, ic, t_end, eps=1e-6, maxsteps=100000):
        hs = np.zeros(maxsteps)
        n = self.L.orc_record_steps(p.h, np.ascontiguousarray(ic, np.float64), eps, t_end, maxsteps, hs)
        if n < 0:
            raise RuntimeError("step recording failed (underflow or too many steps)")
        return hs[:n].copy()

    @staticmethod
    def _wptr(w):
        if w is None:
            return None, None
        w = np.ascontiguousarray(w, np.float64)
        return w, w.ctypes.data_as(C.c_void_p)

    def fixed_loss(self, p, x0, hs, w=None):
        w, wp = self._wptr(w)
        return self.L.orc_fixed_loss(p.h, np.ascontiguousarray(x0, np.float64), wp,
                                     np.ascontiguousarray(hs, np.float64), len(hs), None)

    def adjoint(self, p, x0, hs, w=None):
        w, wp = self._wptr(w)
        gx = np.zeros(p.n + p.m)
        gw = np.zeros(p.m)
        L = self.L.orc_adjoint(p.h, np.ascontiguousarray(x0, np.float64), wp,
                               np.ascontiguousarray(hs, np.float64), len(hs), gx, gw)
        return L, gx, gw

    def potential(self, p, x, w=None):
        wp = None
        if w is not None:
            w = np.ascontiguousarray(w, np.float64)
            wp = w.ctypes.data_as(C.c_void_p)
        return self.L.orc_potential(p.h, np.ascontiguousarray(x, np.float64), wp)


class Reference:
    """The reference AnalogSAT CPU solver + MiniSat built from its sources."""

    KIND = {"random": 0, "planted": 1, "fast": 2}

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference checker not built: {path}")
        L = C.CDLL(path)
        L.refp_from_arrays.restype = C.c_void_p
        L.refp_from_arrays.argtypes = [_i32p, _i32p, C.c_int]
        L.refp_make.restype = C.c_void_p
        L.refp_make.argtypes = [C.c_int, C.c_ulong, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.refp_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3
        L.refp_nlits.restype = C.c_int
        L.refp_nlits.argtypes = [C.c_void_p]
        L.refp_export.argtypes = [C.c_void_p, _i32p, _i32p]
        L.refp_write_cnf.restype = C.c_int
        L.refp_write_cnf.argtypes = [C.c_void_p, C.c_char_p]
        L.refp_read_cnf.restype = C.c_void_p
        L.refp_read_cnf.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.refp_free.argtypes = [C.c_void_p]
        L.ref_rhs_d.restype = C.c_int
        L.ref_rhs_d.argtypes = [C.c_void_p, _f64p, _f64p]
        L.ref_rhs_f.restype = C.c_int
        L.ref_rhs_f.argtypes = [C.c_void_p, _f32p, _f32p]
        L.ref_violations_d.restype = C.c_int
        L.ref_violations_d.argtypes = [C.c_void_p, _f64p]
        L.ref_steps_d.restype = C.c_int
        L.ref_steps_d.argtypes = [C.c_void_p, _f64p, C.c_double, C.c_int, _f64p, _f64p, _i32p,
                                  _i32p, _f64p]
        L.ref_steps_f.restype = C.c_int
        L.ref_steps_f.argtypes = [C.c_void_p, _f32p, C.c_float, C.c_int, _f64p, _f64p, _i32p,
                                  _i32p, _f32p]
        L.ref_solve_d.restype = C.c_int
        L.ref_solve_d.argtypes = [C.c_void_p, _f64p, C.c_double, C.c_double, C.c_int, C.c_int,
                                  _f64p, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.ref_solve_many_d.restype = C.c_int
        L.ref_solve_many_d.argtypes = [C.POINTER(C.c_void_p), _i32p, _f64p, _i64p, C.c_int,
                                       C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                       C.c_double, _i32p, _i32p, _i32p, _f64p, _i32p, _f64p,
                                       C.POINTER(C.c_double)]
        L.ref_minisat.restype = C.c_int
        L.ref_minisat.argtypes = [C.c_void_p, C.c_void_p]
        L.ref_set_model.restype = None
        L.ref_set_model.argtypes = [C.c_int, C.c_double, C.c_double]
        self.L = L

    def set_model(self, tanh=False, q=1.1, b=0.0):
        """CTDS variant of every following call: CpuSatTanh (slope q) or CpuSat, Set_B(b)."""
        self.L.ref_set_model(int(tanh), float(q), float(b))

    class Problem:
        def __init__(self, L, h, planted=None):
            self.L, self.h, self.planted = L, h, planted
            n, m, k = C.c_int(), C.c_int(), C.c_int()
            L.refp_info(h, C.byref(n), C.byref(m), C.byref(k))
            self.n, self.m, self.k = n.value, m.value, k.value

        def export(self):
            nl = self.L.refp_nlits(self.h)
            lits = np.zeros(nl, np.int32)
            lens = np.zeros(self.m, np.int32)
            self.L.refp_export(self.h, lits, lens)
            return lits, lens

        def __del__(self):
            try:
                self.L.refp_free(self.h)
            except Exception:
                pass

    def make(self, kind, seed, n, m, k):
        planted = np.zeros(n, np.int32)
        h = self.L.refp_make(self.KIND[kind], seed, n, m, k, planted.ctypes.data_as(C.c_void_p))
        return Reference.Problem(self.L, h, planted if kind == "planted" else None)

    def problem(self, lits, lens):
        h = self.L.refp_from_arrays(np.ascontiguousarray(lits, np.int32),
                                    np.ascontiguousarray(lens, np.int32), len(lens))
        return Reference.Problem(self.L, h)

    def write_cnf(self, p, path):
        return self.L.refp_write_cnf(p.h, path.encode())

    def read_cnf(self, path):
        msg = C.create_string_buffer(256)
        h = self.L.refp_read_cnf(path.encode(), msg, 256)
        if not h:
            raise ValueError(msg.value.decode())
        return Reference.Problem(self.L, h)

    def rhs(self, p, x, dtype=np.float64):
        if dtype == np.float32:
            x = np.ascontiguousarray(x, np.float32)
            d = np.zeros(p.n + p.m, np.float32)
            assert self.L.ref_rhs_f(p.h, x, d) == 0
            return d
        x = np.ascontiguousarray(x, np.float64)
        d = np.zeros(p.n + p.m, np.float64)
        assert self.L.ref_rhs_d(p.h, x, d) == 0
        return d

    def violations(self, p, x):
        full = np.zeros(p.n + p.m)
        full[: len(x)] = x
        return self.L.ref_violations_d(p.h, full)

    def steps(self, p, ic, eps, nsteps, dtype=np.float64):
        nm = p.n + p.m
        t = np.zeros(nsteps); h = np.zeros(nsteps)
        r = np.zeros(nsteps, np.int32); a = np.zeros(nsteps, np.int32)
        if dtype == np.float32:
            st = np.zeros(nsteps * nm, np.float32)
            done = self.L.ref_steps_f(p.h, np.ascontiguousarray(ic, np.float32), eps, nsteps,
                                      t, h, r, a, st)
        else:
            st = np.zeros(nsteps * nm)
            done = self.L.ref_steps_d(p.h, np.ascontiguousarray(ic, np.float64), eps, nsteps,
                                      t, h, r, a, st)
        return dict(n=done, time=t[:done], h=h[:done], rhs=r[:done], attempts=a[:done],
                    states=st.reshape(nsteps, nm)[:done])

    def solve(self, p, ic, eps=1e-6, tmax=1e8, maxsteps=50_000_000, batch=50):
        fin = np.zeros(p.n + p.m)
        t = C.c_double(); st = C.c_int(); r = C.c_int(); v = C.c_int(); w = C.c_double()
        res = self.L.ref_solve_d(p.h, np.ascontiguousarray(ic, np.float64), eps, tmax, maxsteps,
                                 batch, fin, C.byref(t), C.byref(st), C.byref(r), C.byref(v),
                                 C.byref(w))
        return dict(result=res, state=fin, time=t.value, steps=st.value, rhs=r.value,
                    violations=v.value, wall=w.value)

    def solve_many(self, problems, prob_idx, ics, eps=1e-6, tmax=1e8, maxsteps=50_000_000,
                   batch=50, nthreads=None, wall_budget=0.0):
        """Units u = (problems[prob_idx[u]], ics[u]) over nthreads host threads."""
        nthreads = nthreads or os.cpu_count() or 1
        handles = (C.c_void_p * len(problems))(*[p.h for p in problems])
        prob_idx = np.ascontiguousarray(prob_idx, np.int32)
        n = len(prob_idx)
        flat = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float64) for x in ics]))
        offs = np.zeros(n, np.int64)
        if n > 1:
            offs[1:] = np.cumsum([len(x) for x in ics])[:-1]
        res = np.full(n, -1, np.int32); st = np.zeros(n, np.int32); rh = np.zeros(n, np.int32)
        tm = np.zeros(n); done = np.zeros(n, np.int32); busy = np.zeros(n); wall = C.c_double()
        comp = self.L.ref_solve_many_d(handles, prob_idx, flat, offs, n, nthreads, eps, tmax,
                                       maxsteps, batch, wall_budget, res, st, rh, tm, done, busy,
                                       C.byref(wall))
        return dict(completed=comp, result=res, steps=st, rhs=rh, time=tm, done=done,
                    busy=busy, wall=wall.value, threads=nthreads)

    def minisat(self, p):
        sol = np.zeros(max(p.n, 1), np.int32)
        code = self.L.ref_minisat(p.h, sol.ctypes.data_as(C.c_void_p))
        return code, sol[: p.n]


class RefCuda:
    """The reference's own CUDA path (CudaSat1 + CudaRungeKutta via SatSolver, one
    instance and one trajectory per solver) built for sm_100a: the plain GPU path."""

    def __init__(self, path: str = REFCUDA_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference CUDA comparator not built: {path}")
        L = C.CDLL(path)
        L.refcuda_solve_many.restype = C.c_int
        L.refcuda_solve_many.argtypes = [
            C.c_int, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), _i32p, C.c_int, _i32p,
            _f64p, _i64p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, _i32p, _i32p, _i32p,
            _f64p, C.POINTER(C.c_double)]
        self.L = L

    def solve_many(self, problems, prob_idx, ics, precision=1, eps=1e-6, tmax=1e8,
                   maxsteps=100000, batch=50, wall_budget=0.0):
        """problems: list of (literals, lengths); unit u solves problems[prob_idx[u]] from ics[u]."""
        lits = [np.ascontiguousarray(l, np.int32) for l, _ in problems]
        lens = [np.ascontiguousarray(n, np.int32) for _, n in problems]
        lp = (C.c_void_p * len(lits))(*[a.ctypes.data for a in lits])
        np_ = (C.c_void_p * len(lens))(*[a.ctypes.data for a in lens])
        ms = np.array([len(n) for n in lens], np.int32)
        prob_idx = np.ascontiguousarray(prob_idx, np.int32)
        n = len(prob_idx)
        flat = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float64) for x in ics]))
        offs = np.zeros(n, np.int64)
        if n > 1:
            offs[1:] = np.cumsum([len(x) for x in ics])[:-1]
        res = np.full(n, -1, np.int32); st = np.zeros(n, np.int32); rh = np.zeros(n, np.int32)
        tm = np.zeros(n); wall = C.c_double()
        done = self.L.refcuda_solve_many(precision, len(problems), lp, np_, ms, n, prob_idx, flat, offs,
                                         eps, tmax, maxsteps, batch, wall_budget, res, st, rh, tm,
                                         C.byref(wall))
        return dict(done=done, result=res, steps=st, rhs=rh, time=tm, wall=wall.value)
