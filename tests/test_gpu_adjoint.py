"""Gradients through the RK45 integration (the differentiation configuration:
random 3-SAT N=200, M=850, horizon T=5, gradients of V = sum w a K^2 w.r.t. s(0),
a(0) and per-clause weights).

The GPU adjoint is compared with the FP64 oracle adjoint evaluated on the GPU run's
own frozen step sequence (the oracle adjoint is itself pinned to central finite
differences in tests/test_oracle.py), and directly with central differences.
Tolerances (relative, 2-norm over the gradient vector): FP64 1e-9; FP32 5e-4.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _setup(precision, P=6, seed=0):
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import make_instance, initial_states
    raw = [make_instance("random", 200, 850, 3, seed=100 + i)[:2] for i in range(P)]
    s = SatSolver([SatProblem.from_arrays(l, c) for l, c in raw], precision=precision)
    s.SetEpsilon(1e-6)
    dt = np.float32 if precision == 0 else np.float64
    X = np.concatenate([initial_states(200, 850, 1, seed=seed + i) for i in range(P)]).astype(dt)
    s.SetSatStates(np.arange(P, dtype=np.int32), X)
    w = np.random.default_rng(seed).uniform(0.5, 1.5, size=P * 850)
    return s, raw, X.astype(np.float64), w


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("precision,tol", [(1, 1e-9), (0, 5e-4)])
def test_adjoint_matches_oracle(oracle, precision, tol):
    s, raw, X, w = _setup(precision)
    g = s.Adjoint(5.0, weights=w)
    nm = 200 + 850
    for t, (lits, lens) in enumerate(raw):
        p = oracle.problem(lits, lens)
        hs = g["step_sizes"][t]
        assert len(hs) == g["nsteps"][t] > 10 and abs(hs.sum() - 5.0) < 1e-9
        L, gx, gw = oracle.adjoint(p, X[t], hs, w[t * 850:(t + 1) * 850])
        assert abs(g["loss"][t] - L) <= tol * abs(L)
        assert _rel(g["grad_x0"][t * nm:(t + 1) * nm], gx) <= tol
        assert _rel(g["grad_w"][t * 850:(t + 1) * 850], gw) <= tol


def test_adjoint_fp64_steps_follow_reference_controller(oracle):
    """With w = 1 the forward pass is the reference integrator run to T: its step
    sizes are the oracle's (pinned to the reference) up to the last clamped step."""
    s, raw, X, _ = _setup(1, P=2)
    g = s.Adjoint(5.0)
    for t, (lits, lens) in enumerate(raw):
        hs_ref = oracle.record_steps(oracle.problem(lits, lens), X[t], 5.0)
        np.testing.assert_allclose(g["step_sizes"][t], hs_ref, rtol=1e-9)


def test_adjoint_central_differences(oracle):
    """GPU FP64 gradient against central differences (h = 1e-4) of the frozen-step map
    along random unit directions of x(0) and w."""
    s, raw, X, w = _setup(1, P=1, seed=7)
    g = s.Adjoint(5.0, weights=w)
    p = oracle.problem(*raw[0])
    hs = g["step_sizes"][0]
    rng = np.random.default_rng(3)
    eh = 1e-4
    for _ in range(16):
        d = rng.normal(size=X[0].shape); d /= np.linalg.norm(d)
        fd = (oracle.fixed_loss(p, X[0] + eh * d, hs, w) - oracle.fixed_loss(p, X[0] - eh * d, hs, w)) / (2 * eh)
        assert abs(fd - g["grad_x0"] @ d) <= 1e-5 * max(abs(fd), 1e-3)
        dw = rng.normal(size=w.shape); dw /= np.linalg.norm(dw)
        fd = (oracle.fixed_loss(p, X[0], hs, w + eh * dw) - oracle.fixed_loss(p, X[0], hs, w - eh * dw)) / (2 * eh)
        assert abs(fd - g["grad_w"] @ dw) <= 1e-5 * max(abs(fd), 1e-3)


def test_adjoint_config4_shape_64_directions(oracle):
    """The differentiation configuration at its full shape: 1024 random 3-SAT
    instances N=200, M=850, gradients at T=5 of all of them in one call (FP64 and
    FP32).  Central differences (h = 1e-4) of the frozen-step map along 64 random unit
    directions of x(0) and 64 of w, on four instances spread over the batch (FP64,
    relative 1e-5); FP32 against FP64 over all 1024 (2-norm over every gradient
    entry <= 1e-5, per instance <= 5e-4 for 99% of them)."""
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import make_instance, initial_states
    P, n, m = 1024, 200, 850
    raw = [make_instance("random", n, m, 3, seed=6000 + i)[:2] for i in range(P)]
    X = np.concatenate([initial_states(n, m, 1, seed=60_000 + i) for i in range(P)])
    w = np.random.default_rng(6).uniform(0.5, 1.5, size=P * m)
    probs = [SatProblem.from_arrays(l, c) for l, c in raw]
    g = {}
    for prec, dt in ((1, np.float64), (0, np.float32)):
        s = SatSolver(probs, precision=prec)
        s.SetEpsilon(1e-6)
        s.SetSatStates(np.arange(P, dtype=np.int32), X.astype(dt))
        g[prec] = s.Adjoint(5.0, weights=w)
    nm = n + m
    rng = np.random.default_rng(64)
    eh = 1e-4
    for t in (0, 341, 682, 1023):
        p = oracle.problem(*raw[t])
        hs = g[1]["step_sizes"][t]
        x0, wt = X[t], w[t * m:(t + 1) * m]
        gx, gw = g[1]["grad_x0"][t * nm:(t + 1) * nm], g[1]["grad_w"][t * m:(t + 1) * m]
        for _ in range(64):
            d = rng.normal(size=nm); d /= np.linalg.norm(d)
            fd = (oracle.fixed_loss(p, x0 + eh * d, hs, wt) - oracle.fixed_loss(p, x0 - eh * d, hs, wt)) / (2 * eh)
            assert abs(fd - gx @ d) <= 1e-5 * max(abs(fd), 1e-3), (t, fd, gx @ d)
            dw = rng.normal(size=m); dw /= np.linalg.norm(dw)
            fd = (oracle.fixed_loss(p, x0, hs, wt + eh * dw) - oracle.fixed_loss(p, x0, hs, wt - eh * dw)) / (2 * eh)
            assert abs(fd - gw @ dw) <= 1e-5 * max(abs(fd), 1e-3), (t, fd, gw @ dw)
    for key, size in (("grad_x0", nm), ("grad_w", m)):
        a, b = g[0][key], g[1][key]
        assert _rel(a, b) <= 1e-5, (key, _rel(a, b))
        per = np.array([_rel(a[t * size:(t + 1) * size], b[t * size:(t + 1) * size]) for t in range(P)])
        assert np.quantile(per, 0.99) <= 5e-4, (key, np.quantile(per, 0.99))
