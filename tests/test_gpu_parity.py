"""Parity of the CUDA path (called through the C ABI) with the reference.

Checkers: the golden fixtures written by the reference solver itself
(tests/golden/make_golden.py) and the pinned FP64 C restatement in oracle/.
Tolerances:
  * FP64 RHS / clause counts: bit-exact.
  * FP64 solver vs the oracle: identical accept/reject sequence and counters; states
    within 1e-9 relative (the controller's pow() may differ from glibc by an ulp).
  * FP32 (log-space a) RHS vs FP64: |d32 - d64| <= 1e-5 * max|d64| per vector.
  * FP32 solver vs an FP64 run of the same integrator over a short horizon:
    error <= 1e-5 relative to max(|x|, 1) at equal analog time.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

RHS_TAGS = ["p50", "mix", "r4", "k12", "p200", "p1000"]


def _prob(golden, tag):
    from analogsat_b200 import SatProblem
    return SatProblem.from_arrays(golden[f"{tag}/literals"], golden[f"{tag}/lengths"])


def _cuda(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.mark.parametrize("tag", RHS_TAGS)
def test_rhs_f64_bit_exact(golden, tag):
    from analogsat_b200 import get_derivatives
    p = _prob(golden, tag)
    x = _cuda(golden[f"{tag}/rhs_states"])
    d = get_derivatives(p, x).cpu().numpy()
    ref = golden[f"{tag}/rhs_f64"]
    assert np.array_equal(d, ref), np.abs(d - ref).max()


@pytest.mark.parametrize("tag", RHS_TAGS)
def test_rhs_f32_close(golden, tag):
    from analogsat_b200 import get_derivatives
    p = _prob(golden, tag)
    x = _cuda(golden[f"{tag}/rhs_states"], torch.float32)
    d = get_derivatives(p, x).cpu().numpy().astype(np.float64)
    ref = golden[f"{tag}/rhs_f64"]
    for a, b in zip(d, ref):
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max() + 1e-30


@pytest.mark.parametrize("tag", ["p200", "p1000"])
def test_rhs_logspace(golden, tag):
    from analogsat_b200 import get_derivatives
    p = _prob(golden, tag)
    x = golden[f"{tag}/rhs_states"].copy()
    rng = np.random.default_rng(0)
    x[:, p.n:] = rng.uniform(0.5, 4.0, size=(x.shape[0], p.m))
    d_lin = get_derivatives(p, _cuda(x)).cpu().numpy()
    xl = x.copy()
    xl[:, p.n:] = np.log2(x[:, p.n:])
    d_log = get_derivatives(p, _cuda(xl, torch.float32), logspace=True).cpu().numpy()
    for a, b, xx in zip(d_log, d_lin, x):
        assert np.abs(a[: p.n] - b[: p.n]).max() <= 1e-5 * np.abs(b[: p.n]).max()
        du_ref = b[p.n:] / xx[p.n:] / np.log(2.0)
        assert np.abs(a[p.n:] - du_ref).max() <= 1e-5 * np.abs(du_ref).max() + 1e-30


@pytest.mark.parametrize("tag", RHS_TAGS)
def test_violation_counts_exact(golden, tag):
    from analogsat_b200 import clause_violation_counts
    p = _prob(golden, tag)
    st = golden[f"{tag}/rhs_states"]
    for dt in (torch.float32, torch.float64):
        c = clause_violation_counts(p, _cuda(st, dt)).cpu().numpy()
        assert np.array_equal(c, golden[f"{tag}/viol"])


def test_rhs_and_counts_many_states_vs_oracle(oracle, golden):
    """64 states of the N=1000, M=4250 instance at once, incl. exact zeros and +-1 spins."""
    from analogsat_b200 import get_derivatives, clause_violation_counts
    p = _prob(golden, "p1000")
    op = oracle.problem(golden["p1000/literals"], golden["p1000/lengths"])
    rng = np.random.default_rng(1)
    X = np.concatenate([rng.uniform(-1, 1, (64, p.n)), rng.uniform(0.5, 3, (64, p.m))], axis=1)
    X[0, : p.n] = 0.0
    X[1, : p.n] = np.sign(X[1, : p.n])
    X[2, : p.n] = golden["p1000/planted"] * 2.0 - 1.0
    D = get_derivatives(p, _cuda(X)).cpu().numpy()
    C = clause_violation_counts(p, _cuda(X)).cpu().numpy()
    for i in range(64):
        assert np.array_equal(D[i], oracle.rhs(op, X[i]))
        assert C[i] == oracle.violations(op, X[i])
    assert C[2] == 0  # the planted assignment satisfies every clause


@pytest.mark.parametrize("tag", ["p1000", "r4"])
@pytest.mark.parametrize("logspace", [False, True])
@pytest.mark.parametrize("count,shift,oshift", [(2, 0, 0), (7, 0, 0), (64, 0, 0), (7, 1, 1), (5, 3, 3),
                                                (6, 0, 1), (3, 2, 0)])
def test_rhs_f32_pair_kernel_bit_identical(golden, tag, logspace, count, shift, oshift):
    """FP32 states go through the two-states-per-pass kernel (packed FP32x2, bulk-copied
    row pairs, results in place): each state's derivative is bit-identical whether it
    shares a pass with another state or runs alone (odd counts; state arrays starting
    4, 8 or 12 bytes past a 16-byte boundary; outputs congruent with the inputs mod 16
    bytes, written by bulk stores, or not, written by plain stores)."""
    from analogsat_b200 import get_derivatives
    p = _prob(golden, tag)
    nm = p.n + p.m
    rng = np.random.default_rng(count)
    a = rng.uniform(-1, 2, (count, p.m)) if logspace else rng.uniform(0.5, 3, (count, p.m))
    X = np.concatenate([rng.uniform(-1, 1, (count, p.n)), a], axis=1).astype(np.float32)
    X[0, : p.n] = np.sign(X[0, : p.n])
    flat = torch.zeros(count * nm + 4, dtype=torch.float32, device="cuda")
    xd = flat[shift:shift + count * nm].view(count, nm)
    xd.copy_(torch.from_numpy(X))
    oflat = torch.full((count * nm + 8,), 7.0, dtype=torch.float32, device="cuda")
    out = oflat[oshift:oshift + count * nm].view(count, nm)
    get_derivatives(p, xd, out=out, logspace=logspace)
    D = out.cpu().numpy()
    o = oflat.cpu().numpy()
    assert np.all(o[:oshift] == 7.0) and np.all(o[oshift + count * nm:] == 7.0)  # nothing outside
    assert np.array_equal(xd.cpu().numpy(), X)  # input untouched
    for i in range(count):
        d1 = get_derivatives(p, _cuda(X[i:i + 1], torch.float32), logspace=logspace).cpu().numpy()
        assert np.array_equal(D[i], d1[0]), (i, np.abs(D[i] - d1[0]).max())


def _solver(golden, tag, precision, eps, batch, maxsteps, tmax=1e8):
    from analogsat_b200 import SatSolver
    s = SatSolver([_prob(golden, tag)], precision=precision)
    s.SetEpsilon(eps)
    s.SetBatchSize(batch)
    s.SetMaxSteps(maxsteps)
    s.SetMaxTime(tmax)
    return s


@pytest.mark.parametrize("tag", ["p50", "mix", "r4", "p200"])
def test_solver_f64_matches_oracle(oracle, golden, tag):
    """Same integrator loop as SatSolver::DoSolve with batch 1: counters exact,
    states to 1e-9, against the oracle run with identical parameters."""
    from analogsat_b200 import AS_PREC_F64
    nsteps = len(golden[f"{tag}/traj_time"])
    ic = golden[f"{tag}/traj_ic"]
    s = _solver(golden, tag, AS_PREC_F64, 1e-6, 1, nsteps)
    s.SetSatStates([0], ic[None, :])
    s.Solve()
    r = s.results()
    op = oracle.problem(golden[f"{tag}/literals"], golden[f"{tag}/lengths"])
    o = oracle.solve(op, ic, eps=1e-6, maxsteps=nsteps, batch=1)
    assert r["status"][0] == o["result"]
    assert r["steps"][0] == o["steps"]
    assert r["rhs"][0] == o["rhs"]
    assert r["attempts"][0] == o["attempts"]
    assert r["violations"][0] == o["violations"]
    assert abs(r["time"][0] - o["time"]) <= 1e-9 * o["time"]
    x = s.GetSatState(0)
    np.testing.assert_allclose(x, o["state"], rtol=1e-9, atol=1e-12)
    if o["steps"] == nsteps:  # no early solution: also the reference's own trajectory
        np.testing.assert_allclose(x, golden[f"{tag}/traj_final"], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("tag", ["p50", "cfg1"])
def test_solver_f64_reference_solves(golden, tag):
    """The reference's SatSolver runs (eps 1e-6, batch 50): same SatResult, and every
    solution verified exactly; step counts match while trajectories stay identical."""
    from analogsat_b200 import AS_PREC_F64
    from analogsat_b200.instances import is_satisfied
    eps, batch, maxsteps, tmax = golden[f"{tag}/solve_params"]
    ics = golden[f"{tag}/solve_ics"]
    s = _solver(golden, tag, AS_PREC_F64, eps, int(batch), int(maxsteps), tmax)
    s.SetSatStates(np.zeros(len(ics), np.int32), ics)
    s.Solve()
    r = s.results()
    X = s.GetSatStates().reshape(len(ics), -1)
    n = int(golden[f"{tag}/nmk"][0])
    same = 0
    for i in range(len(ics)):
        assert r["status"][i] == golden[f"{tag}/solve_result"][i]
        if r["status"][i] == 0:
            assert r["violations"][i] == 0
            assert is_satisfied(golden[f"{tag}/literals"], golden[f"{tag}/lengths"], X[i, :n] > 0)
        if r["steps"][i] == golden[f"{tag}/solve_steps"][i]:
            same += 1
    assert same >= len(ics) // 2


@pytest.mark.parametrize("tag,nsteps", [("p200", 40), ("p1000", 30)])
def test_solver_f32_short_horizon_error(oracle, golden, tag, nsteps):
    """FP32 state + log-space a against the FP64 solution of the same ODE at the same
    analog time (oracle integrated to the GPU's end time with eps 1e-10).  FP32 noise
    in the error estimate changes the step sequence, so states are compared at equal
    time, not equal step count.  Bound: 1e-5 relative to max(|x|, 1), i.e. absolute
    for spins (|s| <= 1) and relative for clause weights (a >= 1)."""
    from analogsat_b200 import AS_PREC_F32_LOGA
    ic = golden[f"{tag}/traj_ic"]
    s = _solver(golden, tag, AS_PREC_F32_LOGA, 1e-6, nsteps, nsteps)
    s.SetSatStates([0], ic[None, :])
    s.Solve()
    r = s.results()
    assert r["steps"][0] == nsteps
    op = oracle.problem(golden[f"{tag}/literals"], golden[f"{tag}/lengths"])
    o = oracle.integrate_to(op, ic, r["time"][0], eps=1e-10)
    assert abs(o["time"] - r["time"][0]) <= 1e-12 * r["time"][0]
    x = s.GetSatState(0)
    err = np.abs(x - o["state"]) / np.maximum(np.abs(o["state"]), 1.0)
    assert err.max() <= 1e-5, err.max()


def test_solver_f32_solves_planted_and_verifies():
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import make_instance, initial_states, is_satisfied
    probs, raw = [], []
    for i in range(4):
        lits, lens, _ = make_instance("planted", 1000, 4250, 3, seed=2000 + i)
        raw.append((lits, lens))
        probs.append(SatProblem.from_arrays(lits, lens))
    s = SatSolver(probs)
    s.SetEpsilon(1e-6)
    s.SetBatchSize(50)
    s.SetMaxSteps(200000)
    s.SetMaxTime(1e8)
    T = 8
    pidx = np.repeat(np.arange(4), T).astype(np.int32)
    st = np.concatenate([initial_states(1000, 4250, T, seed=10 + i, dtype=np.float32)
                         for i in range(4)])
    s.SetSatStates(pidx, st)
    s.Solve()
    r = s.results()
    X = s.GetSatStates(np.float32).reshape(len(pidx), -1)
    assert (r["status"] == 0).mean() >= 0.9
    for u in range(len(pidx)):
        if r["status"][u] == 0:
            lits, lens = raw[pidx[u]]
            assert is_satisfied(lits, lens, X[u, :1000] > 0)


def test_solver_deterministic(golden):
    from analogsat_b200 import AS_PREC_F32_LOGA
    ics = golden["p50/solve_ics"]
    outs = []
    for _ in range(2):
        s = _solver(golden, "p50", AS_PREC_F32_LOGA, 1e-6, 50, 200000)
        s.SetSatStates(np.zeros(len(ics), np.int32), ics.astype(np.float32))
        s.Solve()
        outs.append((s.results(), s.GetSatStates(np.float32)))
    for k in outs[0][0]:
        assert np.array_equal(outs[0][0][k], outs[1][0][k])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_limits_and_statuses(golden):
    from analogsat_b200 import AS_PREC_F32_LOGA, SatResult
    ic = golden["p1000/solve_ics"][0:1].astype(np.float32)  # the slow trajectory (22650 steps)
    s = _solver(golden, "p1000", AS_PREC_F32_LOGA, 1e-6, 50, 120)
    s.SetSatStates([0], ic)
    s.Solve()
    r = s.results()
    assert r["status"][0] == SatResult.SAT_MAXITER_REACHED and r["steps"][0] == 150
    s.SetMaxSteps(10 ** 7)
    s.SetMaxTime(0.5)
    s.Solve()
    r = s.results()
    assert r["status"][0] == SatResult.SAT_MAXTIME_REACHED and r["time"][0] >= 0.5
    s.SetMaxTime(1e8)
    s.SetWallBudget(0.05)
    s.Solve()
    r = s.results()
    assert r["status"][0] == SatResult.SAT_ODE_INTERRUPTED or (
        r["status"][0] == SatResult.SAT_SOLUTION_FOUND and r["violations"][0] == 0)


def test_stop_on_first_and_uneven_batch():
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import make_instance, initial_states, is_satisfied
    sizes = [(60, 250), (300, 1270), (1000, 4200), (130, 540)]
    probs, raw = [], []
    for i, (n, m) in enumerate(sizes):
        lits, lens, _ = make_instance("planted", n, m, 3, seed=50 + i)
        raw.append((lits, lens, n))
        probs.append(SatProblem.from_arrays(lits, lens))
    s = SatSolver(probs)
    s.SetEpsilon(1e-6); s.SetBatchSize(20); s.SetMaxSteps(100000); s.SetMaxTime(1e8)
    s.SetStopOnFirst(True)
    T = 16
    pidx = np.repeat(np.arange(len(sizes)), T).astype(np.int32)
    st = np.concatenate([initial_states(n, m, T, seed=i, dtype=np.float32)
                         for i, (n, m) in enumerate(sizes)], axis=None)
    s.SetSatStates(pidx, st)
    s.Solve()
    r = s.results()
    for p in range(len(sizes)):
        sel = pidx == p
        assert (r["status"][sel] == 0).any()
        assert set(r["status"][sel]) <= {0, 2}
        for u in np.nonzero(sel & (r["status"] == 0))[0]:
            x = s.GetSatState(int(u), np.float32)
            lits, lens, n = raw[p]
            assert is_satisfied(lits, lens, x[:n] > 0)


def test_maxsat_best_assignment():
    """Unsatisfiable-w.h.p. instance: min unsat count and the stored best assignment agree."""
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import make_instance, initial_states
    lits, lens, _ = make_instance("random", 80, 640, 3, seed=9)
    p = SatProblem.from_arrays(lits, lens)
    s = SatSolver([p])
    s.SetEpsilon(1e-6); s.SetBatchSize(10); s.SetMaxSteps(3000); s.SetMaxTime(1e8)
    s.SetTrackBest(True)
    s.SetSatStates(np.zeros(4, np.int32), initial_states(80, 640, 4, seed=3, dtype=np.float32))
    s.Solve()
    r = s.results()
    c = lits.reshape(-1, 3)
    for t in range(4):
        best = s.GetBestAssignment(t)
        v = np.abs(c) - 1
        sat = np.where(c > 0, best[v], ~best[v]).any(axis=1)
        assert (~sat).sum() == r["min_violations"][t]
        assert r["min_violations"][t] <= r["violations"][t]


def test_result_file_and_perf_line(golden, tmp_path):
    """The reference frontend's output formats: the MiniSat-compatible result file of a
    solved trajectory (its assignment satisfies the formula) and an unsolved one
    (INDET), and the tab-separated perf line."""
    from analogsat_b200 import SatSolver
    from analogsat_b200.instances import is_satisfied
    p = _prob(golden, "p50")
    s = SatSolver([p], precision=1)
    s.SetEpsilon(1e-6); s.SetBatchSize(50); s.SetMaxSteps(200000); s.SetMaxTime(1e8)
    ics = golden["p50/solve_ics"][:2].copy()
    s.SetSatStates([0, 0], ics)
    s.Solve()
    r = s.results()
    assert r["status"][0] == 0
    out = tmp_path / "p50.out"
    s.WriteResult(0, str(out))
    head, body = out.read_text().splitlines()
    assert head == "SAT"
    lits = [int(t) for t in body.split()]
    assert lits[-1] == 0 and [abs(v) for v in lits[:-1]] == list(range(1, p.n + 1))
    assign = np.array([v > 0 for v in lits[:-1]])
    assert is_satisfied(golden["p50/literals"], golden["p50/lengths"], assign)
    s2 = SatSolver([p], precision=1)
    s2.SetBatchSize(1); s2.SetMaxSteps(1)
    s2.SetSatStates([0], ics[:1])
    s2.Solve()
    s2.WriteResult(0, str(tmp_path / "b.out"))
    assert (tmp_path / "b.out").read_text().splitlines()[0] == "INDET"
    tsv = tmp_path / "perf.tsv"
    s.AppendPerf(0, str(tsv), "p50")
    s.AppendPerf(1, str(tsv), "p50")
    rows = [ln.split("\t") for ln in tsv.read_text().splitlines()]
    assert len(rows) == 2 and all(len(rw) == 7 for rw in rows)
    assert rows[0][0] == "p50" and rows[0][3] == "solution found"
    assert int(rows[0][6]) == r["rhs"][0] and float(rows[0][4]) > 0


@pytest.mark.parametrize("tag", ["p50", "r4", "p200", "p1000"])
def test_lean_kernel_matches_generic_kernel(golden, tag):
    """The lean FP32 kernel (literal words carrying shared-memory byte offsets,
    interleaved RK rows; as_solver_set_kernel) runs the general FP32 kernel's
    integrator and arithmetic: over 8 trajectories and 300 steps the same accepted and
    attempted steps and RHS counts, and states equal to FP32 rounding (relative 1e-6).
    The two launch plans differ (the lean layout's shared-memory size), which shows
    that each kernel ran."""
    from analogsat_b200 import AS_PREC_F32_LOGA, _abi
    n, m, _ = (int(v) for v in golden[f"{tag}/nmk"])
    from analogsat_b200.instances import initial_states
    ics = initial_states(n, m, 8, seed=77, dtype=np.float32)
    out, shapes = {}, {}
    for kern in (_abi.AS_KERNEL_GENERIC, _abi.AS_KERNEL_AUTO):
        s = _solver(golden, tag, AS_PREC_F32_LOGA, 1e-6, 25, 300)
        s.SetKernel(kern)
        s.SetSatStates(np.zeros(8, np.int32), ics)
        s.Solve()
        out[kern] = (s.results(), s.GetSatStates(np.float32).reshape(8, -1))
        shapes[kern] = (s.launch_shape()["smem_bytes"], s.kernel_name())
    (ra, xa), (rb, xb) = out[_abi.AS_KERNEL_GENERIC], out[_abi.AS_KERNEL_AUTO]
    assert shapes[_abi.AS_KERNEL_GENERIC][0] != shapes[_abi.AS_KERNEL_AUTO][0]
    assert shapes[_abi.AS_KERNEL_GENERIC][1] == "solve_kernel"
    assert shapes[_abi.AS_KERNEL_AUTO][1] == "solve_kernel_fast"
    for key in ("status", "steps", "attempts", "rhs", "violations"):
        assert np.array_equal(ra[key], rb[key]), key
    np.testing.assert_allclose(xb, xa, rtol=1e-6, atol=1e-6)
    print(tag, "bit-identical" if np.array_equal(xa, xb) else f"max diff {np.abs(xa - xb).max():.3g}")


@pytest.mark.parametrize("n,m", [(1500, 6375), (3000, 12750)])
def test_lean_kernel_global_rows_matches_generic_kernel(n, m):
    """Instances beyond one SM's shared memory: the lean kernel with its interleaved RK
    rows in a global slab (spins and contribution slots still in shared memory) against
    the general kernel's global-storage mode -- same step, attempt and RHS counts, states
    equal to FP32 rounding -- and the lean kernel is the one chosen by default."""
    from analogsat_b200 import AS_PREC_F32_LOGA, SatProblem, SatSolver, _abi
    from analogsat_b200.instances import make_instance, initial_states
    lits, lens, _ = make_instance("planted", n, m, 3, seed=n)
    p = SatProblem.from_arrays(lits, lens)
    ics = initial_states(n, m, 6, seed=3, dtype=np.float32)
    out, names = {}, {}
    for kern in (_abi.AS_KERNEL_GENERIC, _abi.AS_KERNEL_AUTO):
        s = SatSolver([p], precision=AS_PREC_F32_LOGA)
        s.SetEpsilon(1e-6); s.SetBatchSize(25); s.SetMaxSteps(150); s.SetMaxTime(1e8)
        s.SetKernel(kern)
        s.SetClusterSize(1)  # few trajectories would otherwise take a cluster of CTAs each
        s.SetSatStates(np.zeros(6, np.int32), ics)
        s.Solve()
        out[kern] = (s.results(), s.GetSatStates(np.float32).reshape(6, -1))
        names[kern] = s.kernel_name()
    assert names == {_abi.AS_KERNEL_GENERIC: "solve_kernel", _abi.AS_KERNEL_AUTO: "solve_kernel_fast"}
    (ra, xa), (rb, xb) = out[_abi.AS_KERNEL_GENERIC], out[_abi.AS_KERNEL_AUTO]
    for key in ("status", "steps", "attempts", "rhs", "violations"):
        assert np.array_equal(ra[key], rb[key]), key
    np.testing.assert_allclose(xb, xa, rtol=1e-6, atol=1e-6)
    print(n, "bit-identical" if np.array_equal(xa, xb) else f"max diff {np.abs(xa - xb).max():.3g}")


def test_solvers_of_different_sizes_interleave(golden):
    """Two solvers that launch the same kernel with different shared-memory footprints:
    the large one solves, a small one solves, then the large one solves again -- once
    re-recorded (a setter drops its captured solve) and once launched directly on a
    caller's stream.  A kernel's shared-memory limit is a per-device setting, so the
    small solver must not lower it below what the large one's launches need; both
    repeats give the first run's results."""
    import torch
    from analogsat_b200 import AS_PREC_F32_LOGA
    from analogsat_b200.instances import initial_states

    def make(tag, seed):
        n, m, _ = (int(v) for v in golden[f"{tag}/nmk"])
        s = _solver(golden, tag, AS_PREC_F32_LOGA, 1e-6, 25, 200)
        s.SetSatStates(np.zeros(4, np.int32), initial_states(n, m, 4, seed=seed, dtype=np.float32))
        return s

    big = make("p1000", 91)
    big.Solve()
    first = (big.results(), big.GetSatStates(np.float32))
    small = make("p50", 92)
    small.Solve()
    assert big.launch_shape()["smem_bytes"] > small.launch_shape()["smem_bytes"]
    assert big.kernel_name() == small.kernel_name() == "solve_kernel_fast"
    ics = initial_states(*(int(v) for v in golden["p1000/nmk"][:2]), 4, seed=91, dtype=np.float32)
    for direct in (False, True):
        big.SetMaxSteps(200)  # drops the captured solve
        big.SetSatStates(np.zeros(4, np.int32), ics)
        if direct:
            st = torch.cuda.Stream()
            big.SolveAsync(st.cuda_stream)
            big.Sync()
        else:
            big.Solve()
        again = (big.results(), big.GetSatStates(np.float32))
        for key in ("status", "steps", "rhs"):
            assert np.array_equal(first[0][key], again[0][key]), (direct, key)
        assert np.array_equal(first[1], again[1]), direct
