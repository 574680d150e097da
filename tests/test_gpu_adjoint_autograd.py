"""The device adjoint behind a torch.autograd.Function (test harness only): the loss
L_t = V(x_t(T)) = sum_m w_m a_m(T) K_m(T)^2 of every trajectory as a differentiable
function of x(0) and the clause weights w, with the backward pass supplied by
as_solver_adjoint.

Checks: backward equals the adjoint's gradients weighted by grad_output; directional
derivatives through autograd agree with central differences (h = 1e-4) of the FP64
oracle's loss on the same frozen step sequence; and the gradient tunes the auxiliary
initial weights a(0): a few projected gradient steps with torch.optim lower the loss.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

N, M, T_END = 200, 850, 5.0


class CTDSPotential(torch.autograd.Function):
    """losses (P,) = V(x(T)) per trajectory; x0 (P, N+M) and w (P, M), float64."""

    @staticmethod
    def forward(ctx, x0, w, solver, pidx):
        solver.SetSatStates(pidx, x0.detach().cpu().numpy().reshape(-1))
        g = solver.Adjoint(T_END, weights=w.detach().cpu().numpy().reshape(-1))
        ctx.save_for_backward(torch.from_numpy(g["grad_x0"]).reshape(x0.shape),
                              torch.from_numpy(g["grad_w"]).reshape(w.shape))
        return torch.from_numpy(g["loss"])

    @staticmethod
    def backward(ctx, grad_out):
        gx, gw = ctx.saved_tensors
        return gx * grad_out[:, None], gw * grad_out[:, None], None, None


def _setup(P=2, seed=0):
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import make_instance, initial_states
    raw = [make_instance("random", N, M, 3, seed=500 + i)[:2] for i in range(P)]
    s = SatSolver([SatProblem.from_arrays(l, c) for l, c in raw], precision=1)
    s.SetEpsilon(1e-6)
    x0 = torch.from_numpy(np.concatenate([initial_states(N, M, 1, seed=seed + i) for i in range(P)]))
    w = torch.from_numpy(np.random.default_rng(seed).uniform(0.5, 1.5, size=(P, M)))
    return s, raw, x0, w, np.arange(P, dtype=np.int32)


def test_backward_is_the_weighted_adjoint():
    s, raw, x0, w, pidx = _setup()
    x = x0.clone().requires_grad_(True)
    ww = w.clone().requires_grad_(True)
    loss = CTDSPotential.apply(x, ww, s, pidx)
    coef = torch.tensor([0.7, -1.3], dtype=torch.float64)
    (loss * coef).sum().backward()
    s.SetSatStates(pidx, x0.numpy().reshape(-1))
    g = s.Adjoint(T_END, weights=w.numpy().reshape(-1))
    np.testing.assert_allclose(loss.detach().numpy(), g["loss"], rtol=0, atol=0)
    gx = g["grad_x0"].reshape(2, N + M) * coef.numpy()[:, None]
    gw = g["grad_w"].reshape(2, M) * coef.numpy()[:, None]
    assert np.array_equal(x.grad.numpy(), gx)
    assert np.array_equal(ww.grad.numpy(), gw)


def test_autograd_directional_derivatives_match_central_differences(oracle):
    s, raw, x0, w, pidx = _setup(P=1, seed=3)
    x = x0.clone().requires_grad_(True)
    ww = w.clone().requires_grad_(True)
    loss = CTDSPotential.apply(x, ww, s, pidx)
    gx, gw = torch.autograd.grad(loss.sum(), (x, ww))
    p = oracle.problem(*raw[0])
    s.SetSatStates(pidx, x0.numpy().reshape(-1))
    hs = s.Adjoint(T_END, weights=w.numpy().reshape(-1))["step_sizes"][0]  # the frozen steps
    rng = np.random.default_rng(4)
    eh = 1e-4
    X0, W = x0.numpy()[0], w.numpy()[0]
    for _ in range(8):
        d = rng.normal(size=X0.shape); d /= np.linalg.norm(d)
        fd = (oracle.fixed_loss(p, X0 + eh * d, hs, W) - oracle.fixed_loss(p, X0 - eh * d, hs, W)) / (2 * eh)
        assert abs(fd - float(gx[0].numpy() @ d)) <= 1e-5 * max(abs(fd), 1e-3)
        dw = rng.normal(size=W.shape); dw /= np.linalg.norm(dw)
        fd = (oracle.fixed_loss(p, X0, hs, W + eh * dw) - oracle.fixed_loss(p, X0, hs, W - eh * dw)) / (2 * eh)
        assert abs(fd - float(gw[0].numpy() @ dw)) <= 1e-5 * max(abs(fd), 1e-3)


def test_gradient_tunes_initial_clause_weights():
    """Projected gradient descent on a(0) (kept >= 0.05) with torch.optim.SGD, the
    learning rate set from the first gradient (0.2 / its largest entry): the mean
    potential at T falls step after step."""
    s, raw, x0, w, pidx = _setup(P=2, seed=9)
    a0 = x0[:, N:].clone().requires_grad_(True)
    opt = None
    losses = []
    for _ in range(5):
        x = torch.cat([x0[:, :N], a0], dim=1)
        loss = CTDSPotential.apply(x, w, s, pidx).mean()
        if opt is None:
            (g0,) = torch.autograd.grad(loss, a0, retain_graph=True)
            opt = torch.optim.SGD([a0], lr=0.2 / float(g0.abs().max()))
        opt.zero_grad()
        loss.backward()
        losses.append(float(loss.detach()))
        opt.step()
        with torch.no_grad():
            a0.clamp_(min=0.05)
    assert losses[-1] < losses[0]
    assert all(b <= a * (1 + 1e-12) for a, b in zip(losses, losses[1:])), losses
