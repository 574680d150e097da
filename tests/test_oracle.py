"""The oracle (oracle/ctds_oracle.c) pinned against the reference solver's own outputs.

The golden fixtures were produced by the reference AnalogSAT CPU code itself
(tests/golden/make_golden.py); the C restatement must reproduce them bit for bit
in FP64 (same expression order, no FMA contraction).
"""
import os

import numpy as np
import pytest

from oracle import REF_SO

TAGS_RHS = ["p50", "mix", "r4", "k12", "p200", "p1000"]
TAGS_TRAJ = ["p50", "mix", "r4", "p200", "p1000"]


def _problem(oracle, golden, tag):
    p = oracle.problem(golden[f"{tag}/literals"], golden[f"{tag}/lengths"])
    assert (p.n, p.m, p.k) == tuple(golden[f"{tag}/nmk"])
    return p


@pytest.mark.parametrize("tag", TAGS_RHS)
def test_rhs_bit_exact(oracle, golden, tag):
    p = _problem(oracle, golden, tag)
    for x, ref in zip(golden[f"{tag}/rhs_states"], golden[f"{tag}/rhs_f64"]):
        d = oracle.rhs(p, x)
        assert np.array_equal(d, ref), np.abs(d - ref).max()


@pytest.mark.parametrize("tag", TAGS_RHS)
def test_violation_counts_exact(oracle, golden, tag):
    p = _problem(oracle, golden, tag)
    for x, ref in zip(golden[f"{tag}/rhs_states"], golden[f"{tag}/viol"]):
        assert oracle.violations(p, x) == ref


@pytest.mark.parametrize("tag", TAGS_TRAJ)
def test_trajectory_bit_exact(oracle, golden, tag):
    p = _problem(oracle, golden, tag)
    t = golden[f"{tag}/traj_time"]
    tr = oracle.steps(p, golden[f"{tag}/traj_ic"], float(golden[f"{tag}/traj_eps"][0]), len(t))
    assert tr["n"] == len(t)
    assert np.array_equal(tr["time"], t)
    assert np.array_equal(tr["h"], golden[f"{tag}/traj_h"])
    assert np.array_equal(tr["rhs"], golden[f"{tag}/traj_rhs"])
    assert np.array_equal(tr["attempts"], golden[f"{tag}/traj_attempts"])
    assert np.array_equal(tr["states"][-1], golden[f"{tag}/traj_final"])
    assert np.array_equal(tr["states"][len(t) // 2], golden[f"{tag}/traj_mid"])


@pytest.mark.parametrize("tag", ["p50", "cfg1"])
def test_solve_matches_reference(oracle, golden, tag):
    p = _problem(oracle, golden, tag)
    eps, batch, maxsteps, tmax = golden[f"{tag}/solve_params"]
    for i, ic in enumerate(golden[f"{tag}/solve_ics"]):
        r = oracle.solve(p, ic, eps=eps, tmax=tmax, maxsteps=int(maxsteps), batch=int(batch))
        assert r["result"] == golden[f"{tag}/solve_result"][i]
        assert r["steps"] == golden[f"{tag}/solve_steps"][i]
        assert r["rhs"] == golden[f"{tag}/solve_rhs"][i]
        assert r["time"] == golden[f"{tag}/solve_time"][i]
        assert np.array_equal(r["state"], golden[f"{tag}/solve_final"][i])


def test_solutions_verify_exactly(oracle, golden):
    """Every SAT_SOLUTION_FOUND state satisfies all clauses (exact integer check)."""
    from analogsat_b200.instances import is_satisfied
    for tag in ["p50", "cfg1"]:
        p = _problem(oracle, golden, tag)
        for r, x in zip(golden[f"{tag}/solve_result"], golden[f"{tag}/solve_final"]):
            if r == 0:
                assert oracle.violations(p, x) == 0
                assert is_satisfied(golden[f"{tag}/literals"], golden[f"{tag}/lengths"], x[: p.n] > 0)


def test_planted_and_minisat_certificates(oracle, golden):
    from analogsat_b200.instances import is_satisfied
    for tag in ["p50", "p200", "p1000"]:
        assert is_satisfied(golden[f"{tag}/literals"], golden[f"{tag}/lengths"],
                            golden[f"{tag}/planted"].astype(bool))
    assert golden["p50/minisat"][0] == 10
    assert is_satisfied(golden["cfg1/literals"], golden["cfg1/lengths"],
                        golden["cfg1/minisat_solution"].astype(bool))


def test_logspace_same_ode(oracle, golden):
    """Log-space a is the same ODE: du/dt = K^2 = (da/dt)/a, ds/dt unchanged."""
    p = _problem(oracle, golden, "p200")
    x = golden["p200/rhs_states"][0].copy()
    x[p.n:] = np.linspace(0.5, 3.0, p.m)
    d = oracle.rhs(p, x)
    xl = x.copy(); xl[p.n:] = np.log(x[p.n:])
    dl = oracle.rhs(p, xl, logspace=True)
    np.testing.assert_allclose(dl[: p.n], d[: p.n], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(dl[p.n:], d[p.n:] / x[p.n:], rtol=1e-12, atol=1e-18)


def test_logspace_trajectory_close(oracle, golden):
    """Integrating ln a instead of a changes the discretisation only: over a short
    horizon the two FP64 runs agree to the integration tolerance."""
    p = _problem(oracle, golden, "p200")
    ic = golden["p200/traj_ic"]
    lin = oracle.steps(p, ic, 1e-6, 100)
    lg = oracle.steps(p, ic, 1e-6, 100, logspace=True)
    T = min(lin["time"][-1], lg["time"][-1])
    # compare at matching step count; both integrate the same ODE within eps 1e-6
    assert abs(lin["time"][-1] - lg["time"][-1]) / lin["time"][-1] < 0.05
    assert T > 0


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference checker not built here")
def test_oracle_vs_live_reference(oracle):
    """Fresh instances from the reference makers: RHS and 50 steps bit-exact."""
    from oracle import Reference
    R = Reference()
    rng = np.random.default_rng(5)
    for kind, n, m, k, seed in [("planted", 60, 255, 3, 3), ("random", 33, 140, 4, 4),
                                ("fast", 25, 60, 5, 5)]:
        rp = R.make(kind, seed, n, m, k)
        lits, lens = rp.export()
        op = oracle.problem(lits, lens)
        x = np.concatenate([rng.uniform(-1, 1, rp.n), rng.uniform(1, 2, rp.m)])
        assert np.array_equal(R.rhs(rp, x), oracle.rhs(op, x))
        a = R.steps(rp, x, 1e-6, 50)
        b = oracle.steps(op, x, 1e-6, 50)
        assert np.array_equal(a["states"], b["states"]) and np.array_equal(a["h"], b["h"])


def test_oracle_adjoint_matches_central_differences(oracle):
    """The differentiation configuration's shape (random 3-SAT N=200, M=850, T=5):
    the FP64 discrete adjoint of the frozen-step RK45 map against central finite
    differences (h = 1e-4) along 64 random unit directions of x(0) and of w."""
    from analogsat_b200.instances import make_instance, initial_states
    lits, lens, _ = make_instance("random", 200, 850, 3, seed=4)
    p = oracle.problem(lits, lens)
    x0 = initial_states(200, 850, 1, seed=2)[0]
    hs = oracle.record_steps(p, x0, 5.0)
    rng = np.random.default_rng(0)
    w = rng.uniform(0.5, 1.5, 850)
    L, gx, gw = oracle.adjoint(p, x0, hs, w)
    assert np.isclose(L, oracle.fixed_loss(p, x0, hs, w), rtol=1e-14)
    eh = 1e-4
    errs = []
    for _ in range(64):
        d = rng.normal(size=x0.shape); d /= np.linalg.norm(d)
        fd = (oracle.fixed_loss(p, x0 + eh * d, hs, w) - oracle.fixed_loss(p, x0 - eh * d, hs, w)) / (2 * eh)
        errs.append(abs(fd - gx @ d) / max(abs(fd), 1e-12))
        dw = rng.normal(size=w.shape); dw /= np.linalg.norm(dw)
        fd = (oracle.fixed_loss(p, x0, hs, w + eh * dw) - oracle.fixed_loss(p, x0, hs, w - eh * dw)) / (2 * eh)
        errs.append(abs(fd - gw @ dw) / max(abs(fd), 1e-12))
    assert np.median(errs) < 1e-7 and max(errs) < 1e-4


MODELS = {"tanh": (True, 1.1, 0.0), "tanh_q2_b3": (True, 2.0, 3.0), "bias20": (False, 1.1, 20.0)}


@pytest.mark.parametrize("name", list(MODELS))
@pytest.mark.parametrize("tag", ["p50", "mix", "k12", "r4", "p200"])
def test_model_variants_bit_exact(oracle, golden, golden_models, tag, name):
    """CpuSatTanh (Set_Q) and the bias term (Set_B): the C restatement reproduces the
    reference's RHS vectors and 30 Cash-Karp steps bit for bit."""
    tanh, q, b = MODELS[name]
    p = _problem(oracle, golden, tag)
    oracle.set_model(p, tanh, q, b)
    for x, ref in zip(golden[f"{tag}/rhs_states"], golden_models[f"{tag}/{name}/rhs_f64"]):
        d = oracle.rhs(p, x)
        assert np.array_equal(d, ref), np.abs(d - ref).max()
    if f"{tag}/{name}/traj_time" in golden_models:
        tr = oracle.steps(p, golden[f"{tag}/traj_ic"], 1e-6, 30)
        assert np.array_equal(tr["time"], golden_models[f"{tag}/{name}/traj_time"])
        assert np.array_equal(tr["rhs"], golden_models[f"{tag}/{name}/traj_rhs"])
        assert np.array_equal(tr["states"][-1], golden_models[f"{tag}/{name}/traj_final"])


# Failure-path initial states, injected on the host: a NaN or infinite spin or clause
# weight, every weight infinite or zero, and negative weights, whose dynamics blow up
# in finite time so that the step size underflows (SAT_UNDERFLOW, CpuRungeKutta.cpp:
# 246-248, SatSolver.h:322).  Also the smallest epsilon SetEpsilon accepts (1e-16).
FAILURE_CASES = {
    "nan_spin": (3, np.nan), "inf_spin": (3, np.inf), "neg_inf_weight": (60, -np.inf),
    "nan_weight": (60, np.nan), "inf_weights": (slice(50, None), np.inf),
    "zero_weights": (slice(50, None), 0.0), "negative_weights": (slice(50, None), -1.0),
}


def failure_ic(golden, case):
    x = golden["p50/solve_ics"][0].copy()
    where, val = FAILURE_CASES[case]
    x[where] = val
    return x


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference checker not built here")
@pytest.mark.parametrize("case", sorted(FAILURE_CASES) + ["eps_1e-16"])
def test_oracle_failure_paths_vs_live_reference(oracle, golden, case):
    """The oracle reproduces the reference solver's SatResult, counters, time and final
    state on the failure-path inputs (the reference's NaN handling included: fmax
    skips NaN error ratios, CpuRungeKutta.cpp:236)."""
    from oracle import Reference
    R = Reference()
    lits, lens = golden["p50/literals"], golden["p50/lengths"]
    rp, op = R.problem(lits, lens), oracle.problem(lits, lens)
    eps = 1e-16 if case == "eps_1e-16" else 1e-6
    x = golden["p50/solve_ics"][0] if case == "eps_1e-16" else failure_ic(golden, case)
    a = R.solve(rp, x, eps=eps, maxsteps=20000, batch=50, tmax=1e8)
    b = oracle.solve(op, x, eps=eps, maxsteps=20000, batch=50, tmax=1e8)
    for k in ("result", "steps", "rhs", "violations", "time"):
        assert a[k] == b[k], (case, k, a[k], b[k])
    assert np.array_equal(a["state"], b["state"], equal_nan=True)
    if case == "negative_weights":
        assert a["result"] == 1  # SAT_UNDERFLOW


def test_minisat_fixture_certificates():
    """The MiniSat verdict fixture (tests/golden/make_golden_stats.py): every SAT verdict
    carries a model that satisfies its instance exactly; both verdicts occur."""
    from analogsat_b200.instances import is_satisfied
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "minisat_3sat.npz")))
    n, m, k = (int(v) for v in d["nmk"])
    assert set(np.unique(d["verdict"])) == {10, 20}
    for i, v in enumerate(d["verdict"]):
        if v == 10:
            assert is_satisfied(d["literals"][i].astype(np.int32), np.full(m, k, np.int32),
                                d["model"][i].astype(bool))
