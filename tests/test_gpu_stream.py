"""The streamed solver (storage mode 3): eight trajectories per lane group, state
interleaved in device memory, one RK attempt per pass of per-stage kernels.

Checks: in FP64 (explicitly rounded arithmetic) every lane follows exactly the
trajectory of the one-CTA shared-memory solver on the same packing: results and final
states bit-identical, exact-length and mixed-length clauses, k > 10, padded groups,
two problems in one solver.  In FP32 the per-element arithmetic is the same but the
compiler's FMA contraction may differ between the two kernels, so FP32 is checked
against the FP64 solution of the same ODE at equal time (<= 1e-5 relative to
max(|x|, 1)).  Then the SatSolver status rules (max steps, max time, wall-clock
budget), exact solutions and tracked best assignments (re-counted on the host).
"""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _solver(problems, precision, eps=1e-6, batch=20, maxsteps=2000, tmax=1e8):
    from analogsat_b200 import SatSolver
    s = SatSolver(problems, precision=precision)
    s.SetEpsilon(eps)
    s.SetBatchSize(batch)
    s.SetMaxSteps(maxsteps)
    s.SetMaxTime(tmax)
    return s


def _run(problems, precision, pidx, ics, mode, **kw):
    s = _solver(problems, precision, **kw)
    s.SetStorageMode(mode)
    s.SetSatStates(np.asarray(pidx, np.int32), ics)
    s.Solve()
    dt = np.float32 if precision == 0 else np.float64
    return s.results(), s.GetSatStates(dt)


def _same(ref, got):
    for key in ref[0]:
        assert np.array_equal(ref[0][key], got[0][key]), (key, ref[0][key], got[0][key])
    assert np.array_equal(ref[1], got[1])


def test_stream_f64_matches_shared_memory_solver():
    """6 trajectories: one full lane group and one group with two padding lanes."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m, T = 200, 850, 6
    lits, lens, _ = make_instance("planted", n, m, 3, seed=31)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, T, seed=4)
    _same(_run([p], 1, np.zeros(T), ics, 1, batch=7, maxsteps=300),
          _run([p], 1, np.zeros(T), ics, 3, batch=7, maxsteps=300))


@pytest.mark.parametrize("tag", ["mix", "k12", "r4"])
def test_stream_f64_matches_shared_memory_solver_golden(golden, tag):
    """Golden instances: mixed clause lengths (sentinel literals), k = 12 (the generic
    leave-one-out form), 4-SAT; two problems in one solver."""
    from analogsat_b200 import SatProblem
    p = SatProblem.from_arrays(golden[f"{tag}/literals"], golden[f"{tag}/lengths"])
    q = SatProblem.from_arrays(golden["p50/literals"], golden["p50/lengths"])
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-1, 1, (3, p.n)), np.ones((3, p.m))], axis=1)
    ics = np.concatenate([xs.reshape(-1), golden["p50/solve_ics"][:2].reshape(-1)])
    pidx = [0, 0, 0, 1, 1]
    _same(_run([p, q], 1, pidx, ics, 1, batch=5, maxsteps=120),
          _run([p, q], 1, pidx, ics, 3, batch=5, maxsteps=120))


@pytest.mark.parametrize("parts", [1, 3])
def test_stream_f64_wide_instance_matches_global_storage(parts):
    """N=6000, M=25500 (wide literal words, public clause order): the stream solver,
    with its clauses in one part or split into three parts whose row sums continue
    from part to part, against the global-storage solver, bit for bit."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m, T = 6000, 25500, 5
    lits, lens, _ = make_instance("planted", n, m, 3, seed=8)
    p = SatProblem.from_arrays(lits, lens)
    assert not p.layout_stats(1)["compact"]
    ics = initial_states(n, m, T, seed=5)
    ref = _run([p], 1, np.zeros(T), ics, 2, batch=6, maxsteps=60)
    s = _solver([p], 1, batch=6, maxsteps=60)
    s.SetStorageMode(3)
    s.SetStreamParts(parts)
    s.SetSatStates(np.zeros(T, np.int32), ics)
    s.Solve()
    _same(ref, (s.results(), s.GetSatStates(np.float64)))


def test_stream_f32_short_horizon_error(oracle):
    """FP32 stream lanes against the FP64 solution of the ODE at the same time."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m, T = 1000, 4250, 4
    lits, lens, _ = make_instance("planted", n, m, 3, seed=2000)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, T, seed=3, dtype=np.float32)
    r, X = _run([p], 0, np.zeros(T), ics, 3, batch=30, maxsteps=30)
    assert (r["status"] == 4).all() and (r["steps"] == 30).all()
    X = X.reshape(T, n + m).astype(np.float64)
    op = oracle.problem(lits, lens)
    for u in range(T):
        o = oracle.integrate_to(op, ics[u].astype(np.float64), r["time"][u], eps=1e-10)
        err = np.abs(X[u] - o["state"]) / np.maximum(np.abs(o["state"]), 1.0)
        assert err.max() <= 1e-5, (u, err.max())


def test_stream_status_rules():
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m = 100, 426
    lits, lens, _ = make_instance("random", n, m, 3, seed=3)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, 4, seed=1)
    for kw, status in ((dict(tmax=1e-12), 3), (dict(maxsteps=3, batch=5), 4), (dict(maxsteps=10, batch=5), 4)):
        ref = _run([p], 1, np.zeros(4), ics, 1, **kw)
        got = _run([p], 1, np.zeros(4), ics, 3, **kw)
        _same(ref, got)
        assert (got[0]["status"] == status).all(), (kw, got[0]["status"])
    assert (got[0]["steps"] == 10).all()


def test_stream_solves_and_tracks_best():
    """Planted N=2000 instance to solution (exact check) with stop on the first
    solution; tracked best assignments re-count to the reported minimum."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states, is_satisfied
    n, m, T = 2000, 8500, 8
    lits, lens, _ = make_instance("planted", n, m, 3, seed=44)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, T, seed=8, dtype=np.float32)
    s = _solver([p], 0, batch=50, maxsteps=100000)
    s.SetStorageMode(3)
    s.SetTrackBest(True)
    s.SetStopOnFirst(True)
    s.SetSatStates(np.zeros(T, np.int32), ics)
    s.Solve()
    r = s.results()
    assert (r["status"] == 0).any()
    assert set(r["status"]) <= {0, 2}
    X = s.GetSatStates(np.float32).reshape(T, n + m)
    c = lits.reshape(-1, 3)
    v = np.abs(c) - 1
    for u in range(T):
        if r["status"][u] == 0:
            assert is_satisfied(lits, lens, X[u, :n] > 0)
        best = s.GetBestAssignment(u)
        assert int((~np.where(c > 0, best[v], ~best[v]).any(axis=1)).sum()) == r["min_violations"][u]


def test_stream_wall_budget():
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m = 20000, 200000
    lits, lens, _ = make_instance("fast", n, m, 4, seed=9)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, 4, seed=2, dtype=np.float32)
    s = _solver([p], 0, batch=10, maxsteps=10 ** 9, tmax=1e30)
    s.SetStorageMode(3)
    s.SetWallBudget(1.0)
    s.SetSatStates(np.zeros(4, np.int32), ics)
    t0 = time.perf_counter()
    s.Solve()
    wall = time.perf_counter() - t0
    r = s.results()
    assert (r["status"] == 2).all()
    assert wall < 10.0
    assert (r["steps"] > 0).all()


def test_stream_f32_error_at_maxsat_size(oracle):
    """The MAXSAT configuration's size (random 4-SAT N=1e5, M=1e6): an FP32 streamed
    trajectory after 40 accepted steps against the FP64 oracle's solution of the same
    ODE at the same time (eps 1e-10), <= 1e-5 relative to max(|x|, 1)."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m = 100_000, 1_000_000
    lits, lens, _ = make_instance("fast", n, m, 4, seed=5000)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, 1, seed=3, dtype=np.float32)
    r, X = _run([p], 0, np.zeros(1), ics, 3, batch=10, maxsteps=40)
    assert r["steps"][0] == 40
    o = oracle.integrate_to(oracle.problem(lits, lens), ics[0].astype(np.float64), r["time"][0], eps=1e-10)
    err = np.abs(X.astype(np.float64) - o["state"]) / np.maximum(np.abs(o["state"]), 1.0)
    print(f"N=1e5/M=1e6 FP32 stream vs FP64 oracle at t={r['time'][0]:.4g}: max rel err {err.max():.3g}")
    assert err.max() <= 1e-5, err.max()
