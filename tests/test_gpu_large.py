"""Large instances: the global-storage path (per-CTA slab in device memory, wide
literal words) for instances that do not fit one SM's shared memory -- the uneven
batch's N up to 5000 and the N=1e5, M=1e6 MAXSAT instance.

Checks: the global-storage solver reproduces the shared-memory solver bit for bit on
an instance both can hold (same arithmetic in the same order, only the storage
differs); the wide-encoding RHS is bit-exact against the oracle in FP64; large-instance
solves verify exactly; the N=1e5 instance runs through RHS, clause count and solver.
"""
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


@pytest.mark.parametrize("precision", [0, 1])
def test_global_storage_matches_shared_memory(precision):
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m, T = 200, 850, 24
    lits, lens, _ = make_instance("planted", n, m, 3, seed=31)
    p = SatProblem.from_arrays(lits, lens)
    dt = np.float32 if precision == 0 else np.float64
    ics = initial_states(n, m, T, seed=4, dtype=dt)
    out = []
    for mode in (1, 2):
        s = _solver([p], precision)
        s.SetStorageMode(mode)
        s.SetSatStates(np.zeros(T, np.int32), ics)
        s.Solve()
        out.append((s.results(), s.GetSatStates(dt)))
    for key in out[0][0]:
        assert np.array_equal(out[0][0][key], out[1][0][key]), key
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("cl", [4, 8])
def test_cluster_storage_matches_single_cta(cl):
    """A trajectory spread over a thread-block cluster (cluster barriers, distributed
    shared memory reductions) gives bit-identical results to one CTA per trajectory."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m, T = 2500, 10625, 6
    lits, lens, _ = make_instance("planted", n, m, 3, seed=21)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, T, seed=9, dtype=np.float32)
    out = []
    for c in (1, cl):
        s = _solver([p], 0, batch=20, maxsteps=400)
        s.SetStorageMode(2)
        s.SetClusterSize(c)
        s.SetSatStates(np.zeros(T, np.int32), ics)
        s.Solve()
        assert s.launch_shape()["ctas"] % c == 0
        out.append((s.results(), s.GetSatStates(np.float32)))
    for key in out[0][0]:
        assert np.array_equal(out[0][0][key], out[1][0][key]), key
    assert np.array_equal(out[0][1], out[1][1])


def test_large_instance_rhs_and_counts(oracle):
    """N=6000, M=25500: beyond the compact encoding (more than 65535 slots)."""
    from analogsat_b200 import SatProblem, get_derivatives, clause_violation_counts
    from analogsat_b200.instances import make_instance
    n, m = 6000, 25500
    lits, lens, planted = make_instance("planted", n, m, 3, seed=8)
    p = SatProblem.from_arrays(lits, lens)
    assert not p.layout_stats(1)["compact"]
    op = oracle.problem(lits, lens)
    rng = np.random.default_rng(2)
    X = np.concatenate([rng.uniform(-1, 1, (3, n)), rng.uniform(0.5, 3, (3, m))], axis=1)
    X[2, :n] = planted * 2.0 - 1.0
    D = get_derivatives(p, torch.tensor(X, device="cuda")).cpu().numpy()
    C = clause_violation_counts(p, torch.tensor(X, device="cuda")).cpu().numpy()
    D32 = get_derivatives(p, torch.tensor(X, dtype=torch.float32, device="cuda")).cpu().numpy()
    for i in range(3):
        ref = oracle.rhs(op, X[i])
        assert np.array_equal(D[i], ref)
        assert np.abs(D32[i] - ref).max() <= 1e-5 * np.abs(ref).max()
        assert C[i] == oracle.violations(op, X[i])
    assert C[2] == 0


def test_large_instance_solve_verifies(oracle):
    """N=3000, M=12750 (global storage): solutions verify exactly, and a short FP32
    horizon agrees with the FP64 solution of the ODE at the same time."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states, is_satisfied
    n, m, T = 3000, 12750, 8
    lits, lens, _ = make_instance("planted", n, m, 3, seed=12)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, T, seed=6, dtype=np.float32)
    s = _solver([p], 0, batch=50, maxsteps=60000)
    s.SetStopOnFirst(True)
    s.SetSatStates(np.zeros(T, np.int32), ics)
    s.Solve()
    r = s.results()
    assert (r["status"] == 0).any()
    X = s.GetSatStates(np.float32).reshape(T, n + m)
    for u in np.nonzero(r["status"] == 0)[0]:
        assert is_satisfied(lits, lens, X[u, :n] > 0)

    h = _solver([p], 0, batch=25, maxsteps=25)
    h.SetSatStates([0], ics[:1])
    h.Solve()
    rh = h.results()
    op = oracle.problem(lits, lens)
    o = oracle.integrate_to(op, ics[0].astype(np.float64), rh["time"][0], eps=1e-10)
    x = h.GetSatState(0, np.float32).astype(np.float64)
    err = np.abs(x - o["state"]) / np.maximum(np.abs(o["state"]), 1.0)
    assert err.max() <= 1e-5, err.max()


def test_maxsat_scale_instance_runs(oracle):
    """The N=1e5, M=1e6 random 4-SAT shape: RHS (FP32 vs FP64 oracle), exact clause
    counts, and a few solver steps whose reported unsat counts are exact."""
    from analogsat_b200 import SatProblem, SatSolver, get_derivatives, clause_violation_counts
    from analogsat_b200.instances import make_instance, initial_states
    n, m, k = 100_000, 1_000_000, 4
    lits, lens, _ = make_instance("fast", n, m, k, seed=5)
    p = SatProblem.from_arrays(lits, lens)
    op = oracle.problem(lits, lens)
    X = initial_states(n, m, 2, seed=1)
    D = get_derivatives(p, torch.tensor(X, dtype=torch.float32, device="cuda")).cpu().numpy()
    C = clause_violation_counts(p, torch.tensor(X, device="cuda")).cpu().numpy()
    for i in range(2):
        ref = oracle.rhs(op, X[i])
        assert np.abs(D[i] - ref).max() <= 1e-5 * np.abs(ref).max()
        assert C[i] == oracle.violations(op, X[i])
    s = SatSolver([p])
    s.SetEpsilon(1e-6); s.SetBatchSize(2); s.SetMaxSteps(4); s.SetMaxTime(1e8)
    s.SetTrackBest(True)
    s.SetSatStates(np.zeros(2, np.int32), X.astype(np.float32))
    s.Solve()
    r = s.results()
    assert list(r["status"]) == [4, 4] and list(r["steps"]) == [4, 4]
    fin = s.GetSatStates(np.float32).reshape(2, n + m)
    for i in range(2):
        assert r["violations"][i] == oracle.violations(op, fin[i].astype(np.float64))
        best = s.GetBestAssignment(i)
        assert oracle.violations(op, np.where(best, 1.0, -1.0)) == r["min_violations"][i]


def test_lean_kernel_in_two_clause_parts_vs_fp64(oracle):
    """N=4800, M=20400: the contribution slots of the whole instance (about 245 KB) do not fit
    one SM, so the lean kernel's global-rows form splits every RHS into two clause parts
    that reuse one slot buffer, the sums continuing from part to part.  FP32 against the
    FP64 solution of the same ODE at the same analog time (oracle at eps 1e-10): 1e-5
    relative to max(|x|, 1), as for the other FP32 paths."""
    from analogsat_b200 import SatProblem
    from analogsat_b200.instances import make_instance, initial_states
    n, m = 4800, 20400
    lits, lens, _ = make_instance("planted", n, m, 3, seed=48)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, 3, seed=5, dtype=np.float32)
    s = _solver([p], 0, eps=1e-6, batch=20, maxsteps=20)
    s.SetClusterSize(1)
    s.SetSatStates(np.zeros(3, np.int32), ics)
    s.Solve()
    assert s.kernel_name() == "solve_kernel_fast"
    # the whole instance's slots exceed one SM; the launch holds one part's
    assert 4 * p.layout_stats()["nslots"] > 227 * 1024 >= s.launch_shape()["smem_bytes"]
    r = s.results()
    X = s.GetSatStates(np.float32).reshape(3, n + m)
    op = oracle.problem(lits, lens)
    for t in range(3):
        assert r["steps"][t] == 20
        o = oracle.integrate_to(op, ics[t].astype(np.float64), r["time"][t], eps=1e-10)
        err = np.abs(X[t] - o["state"]) / np.maximum(np.abs(o["state"]), 1.0)
        assert err.max() <= 1e-5, err.max()
