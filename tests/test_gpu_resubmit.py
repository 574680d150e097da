"""Re-submitting trajectories to a solver: a second as_solver_set_states_* call with
the same trajectory -> problem map keeps the unit tables and the captured solve, so
it must still solve the new values (not the old ones); a changed map rebuilds them.
One-trajectory state reads equal the slices of the full read."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _setup(precision):
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance
    probs = [SatProblem.from_arrays(*make_instance("planted", 150, 630, 3, seed=s)[:2]) for s in (1, 2, 3)]
    return probs


def _solver(probs, precision):
    from analogsat_b200 import SatSolver
    s = SatSolver(probs, precision=precision)
    s.SetEpsilon(1e-6); s.SetBatchSize(10); s.SetMaxSteps(200); s.SetMaxTime(1e8)
    return s


@pytest.mark.parametrize("precision", [0, 1])
def test_same_map_new_values_and_new_map(precision):
    from analogsat_b200.instances import initial_states
    probs = _setup(precision)
    dt = np.float32 if precision == 0 else np.float64
    pidx = np.array([0, 1, 2, 2, 1, 0, 0], np.int32)
    A = initial_states(150, 630, len(pidx), seed=1, dtype=dt)
    B = initial_states(150, 630, len(pidx), seed=2, dtype=dt)
    s = _solver(probs, precision)
    s.SetSatStates(pidx, A); s.Solve()
    s.SetSatStates(pidx, B); s.Solve()   # same map: unit tables and graph kept
    fresh = _solver(probs, precision)
    fresh.SetSatStates(pidx, B); fresh.Solve()
    for key in ("status", "steps", "rhs", "violations"):
        assert np.array_equal(s.results()[key], fresh.results()[key]), key
    assert np.array_equal(s.GetSatStates(dt), fresh.GetSatStates(dt))
    # a different map on the same solver
    q = np.array([2, 2, 0], np.int32)
    C = initial_states(150, 630, 3, seed=3, dtype=dt)
    s.SetSatStates(q, C); s.Solve()
    f2 = _solver(probs, precision)
    f2.SetSatStates(q, C); f2.Solve()
    assert np.array_equal(s.results()["steps"], f2.results()["steps"])
    assert np.array_equal(s.GetSatStates(dt), f2.GetSatStates(dt))
    # one-trajectory reads are the slices of the full read
    full = s.GetSatStates(dt).reshape(3, 780)
    for t in range(3):
        assert np.array_equal(s.GetSatState(t, dt), full[t])


@pytest.mark.parametrize("precision", [0, 1])
def test_solve_async_on_a_caller_stream_then_sync(precision):
    """SolveAsync on a stream of the caller's after a host SetSatStates (queued on the
    solver's own stream), then Sync() and the result reads: the solve starts after the
    states are in place and Sync() returns after it, so the results equal a plain
    Solve() of the same states."""
    from analogsat_b200.instances import initial_states
    probs = _setup(precision)
    dt = np.float32 if precision == 0 else np.float64
    pidx = np.repeat(np.arange(3), 40).astype(np.int32)
    X = initial_states(150, 630, len(pidx), seed=7, dtype=dt)
    ref = _solver(probs, precision)
    ref.SetMaxSteps(3000)
    ref.SetSatStates(pidx, X); ref.Solve()
    side = torch.cuda.Stream()
    for rep in range(2):  # the second round replays with the unit tables kept
        s = _solver(probs, precision) if rep == 0 else s
        s.SetMaxSteps(3000)
        s.SetSatStates(pidx, X)
        s.SolveAsync(stream=side.cuda_stream)
        s.Sync()
        for key in ("status", "steps", "rhs", "violations"):
            assert np.array_equal(s.results()[key], ref.results()[key]), (rep, key)
        assert np.array_equal(s.GetSatStates(dt), ref.GetSatStates(dt))
