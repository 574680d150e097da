"""The reference's CTDS variants on the CUDA path: CpuSatTanh (slope q, Set_Q) and the
bias term (ISat::Set_B), through the C ABI.

Checkers: golden_models.npz (the reference's own RHS vectors) and the pinned FP64
oracle.  Tolerances: the tanh and sine evaluations are CUDA's, not glibc's (a last-
bit difference is allowed), and the bias term's clause-weight sum is reduced in a
different order than the reference's sequential sum, so FP64 is compared within
1e-12 relative to the vector's largest entry instead of bit for bit; FP32 within
1e-5 of FP64 as everywhere; FP64 solver trajectories against the oracle running the
same integrator within 1e-9, FP32 ones against the FP64 solution of the ODE at equal
analog time within 1e-5, both relative to max(|x|, 1).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

MODELS = {"tanh": (True, 1.1, 0.0), "tanh_q2_b3": (True, 2.0, 3.0), "bias20": (False, 1.1, 20.0)}


def _prob(golden, tag, name):
    from analogsat_b200 import SatProblem
    tanh, q, b = MODELS[name]
    p = SatProblem.from_arrays(golden[f"{tag}/literals"], golden[f"{tag}/lengths"])
    p.set_model(tanh, q).set_bias(b)
    return p


def _cuda(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.mark.parametrize("name", list(MODELS))
@pytest.mark.parametrize("tag", ["p50", "mix", "k12", "r4", "p200"])
def test_model_rhs_matches_reference(golden, golden_models, tag, name):
    from analogsat_b200 import get_derivatives
    p = _prob(golden, tag, name)
    assert p.model()["tanh"] == MODELS[name][0]
    X = golden[f"{tag}/rhs_states"]
    ref = golden_models[f"{tag}/{name}/rhs_f64"]
    d64 = get_derivatives(p, _cuda(X)).cpu().numpy()
    d32 = get_derivatives(p, _cuda(X, torch.float32)).cpu().numpy().astype(np.float64)
    for a, b, r in zip(d64, d32, ref):
        scale = np.abs(r).max()
        assert np.abs(a - r).max() <= 1e-12 * scale, np.abs(a - r).max() / scale
        assert np.abs(b - r).max() <= 1e-5 * scale


@pytest.mark.parametrize("name", list(MODELS))
def test_model_rhs_many_states_vs_oracle(oracle, golden, name):
    """64 states of the N=1000/M=4250 instance: the FP32 device RHS with a variant set
    bypasses the two-states-per-pass kernel (plain CTDS only) for the one-state kernel."""
    from analogsat_b200 import get_derivatives
    tanh, q, b = MODELS[name]
    p = _prob(golden, "p1000", name)
    op = oracle.problem(golden["p1000/literals"], golden["p1000/lengths"])
    oracle.set_model(op, tanh, q, b)
    rng = np.random.default_rng(7)
    X = np.concatenate([rng.uniform(-1, 1, (64, p.n)), rng.uniform(0.5, 3, (64, p.m))], axis=1)
    D = get_derivatives(p, _cuda(X)).cpu().numpy()
    D32 = get_derivatives(p, _cuda(X, torch.float32)).cpu().numpy()
    for i in range(0, 64, 7):
        r = oracle.rhs(op, X[i])
        assert np.abs(D[i] - r).max() <= 1e-12 * np.abs(r).max()
        assert np.abs(D32[i] - r).max() <= 1e-5 * np.abs(r).max()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", list(MODELS))
def test_model_solver_short_horizon(oracle, golden, name, precision):
    """Solver (shared-memory and global-storage modes) with a variant, 40 accepted
    steps.  FP64: against the oracle running the same integrator (eps 1e-6, 40 steps).
    FP32: against the FP64 oracle's solution of the same ODE at the same time."""
    from analogsat_b200 import SatSolver
    tanh, q, b = MODELS[name]
    tag = "p200"
    p = _prob(golden, tag, name)
    op = oracle.problem(golden[f"{tag}/literals"], golden[f"{tag}/lengths"])
    oracle.set_model(op, tanh, q, b)
    ic = golden[f"{tag}/traj_ic"]
    dt = np.float32 if precision == 0 else np.float64
    tol = 1e-5 if precision == 0 else 1e-9
    for mode in (1, 2):
        s = SatSolver([p], precision=precision)
        s.SetEpsilon(1e-6); s.SetBatchSize(40); s.SetMaxSteps(40); s.SetMaxTime(1e8)
        s.SetStorageMode(mode)
        s.SetSatStates([0], ic.astype(dt))
        s.Solve()
        r = s.results()
        assert r["steps"][0] == 40
        x = s.GetSatState(0, dt).astype(np.float64)
        if precision == 1:
            tr = oracle.steps(op, ic, 1e-6, 40)
            ref = tr["states"][-1]
            assert abs(r["time"][0] - tr["time"][-1]) <= tol * tr["time"][-1]
        else:
            ref = oracle.integrate_to(op, ic, r["time"][0], eps=1e-10)["state"]
        err = np.abs(x - ref) / np.maximum(np.abs(ref), 1.0)
        assert err.max() <= tol, (mode, err.max())


def test_model_f64_solver_follows_reference_counters(oracle, golden, golden_models):
    """FP64 solver, tanh variant, batch 1: the accepted-step times follow the
    reference's 30 Cash-Karp steps (last-bit tanh differences allowed)."""
    from analogsat_b200 import SatSolver
    tag, name = "p50", "tanh"
    p = _prob(golden, tag, name)
    s = SatSolver([p], precision=1)
    s.SetEpsilon(1e-6); s.SetBatchSize(1); s.SetMaxSteps(30); s.SetMaxTime(1e8)
    s.SetSatStates([0], golden[f"{tag}/traj_ic"])
    s.Solve()
    r = s.results()
    assert r["steps"][0] == 30
    assert r["rhs"][0] == golden_models[f"{tag}/{name}/traj_rhs"][-1]
    assert abs(r["time"][0] - golden_models[f"{tag}/{name}/traj_time"][-1]) <= 1e-9 * r["time"][0]
    x = s.GetSatState(0, np.float64)
    ref = golden_models[f"{tag}/{name}/traj_final"]
    assert np.abs(x - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1.0)


def test_model_unsupported_paths(golden):
    """The streamed solver, thread-block clusters and the adjoint have the plain CTDS
    right-hand side only: they refuse a variant instead of ignoring it."""
    from analogsat_b200 import SatSolver, AnalogSatError
    p = _prob(golden, "p200", "bias20")
    ic = golden["p200/traj_ic"]
    s = SatSolver([p], precision=1)
    s.SetMaxSteps(5); s.SetBatchSize(5)
    s.SetSatStates([0], ic)
    s.SetStorageMode(3)
    with pytest.raises(AnalogSatError):
        s.Solve()
    s.SetStorageMode(2)
    s.SetClusterSize(4)
    with pytest.raises(AnalogSatError):
        s.Solve()
    s.SetClusterSize(0)
    s.Solve()  # automatic: one CTA per trajectory
    with pytest.raises(AnalogSatError):
        s.Adjoint(1.0)
