"""The differentiable traces against central finite differences, in float64.

The adjoint is the exact transpose of the discrete forward step, so the gradient and
the finite difference agree to the difference's own truncation (h^2) and round-off,
as the reference's gradient tests check theirs (cuwave sensitivity_test.py:267-692,
1196-1320: float64 central differences). The cells checked are drawn among those whose
gradient is at least 5% of the largest: elsewhere a difference quotient resolves only the
loss's own round-off.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(mode="history", checkpoints=None, pml=6, ndim=2):
    from cuwave_b200 import AcousticWave, Pml, stable_dt
    from cuwave_b200.autograd import Problem
    from cuwave_b200.signals import ricker

    Nx = (34, 38) if ndim == 2 else (36, 34, 38)
    N = 90 if ndim == 2 else 50
    dt = 0.5 * stable_dt((1.0,) * ndim, 1.3, 8)
    sim = AcousticWave(Nx=Nx, dx=(1.0,) * ndim, N=N, dt=dt, precision="float64", space_order=8,
                       pml=Pml(width=pml, wavespeed=1.3) if pml else None,
                       rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=2.0)
    rng = np.random.default_rng(4)
    src = np.array([[n // 2] for n in Nx], np.int32)
    sens = np.stack([rng.integers(pml + 2, n - pml - 2, 6) for n in Nx]).astype(np.int32)
    c = np.zeros(sim.Nx_padded)
    logical = tuple(slice(0, n) for n in Nx)
    c[logical] = 1.0 + 0.3 * rng.random(Nx)
    signal = ricker(np.arange(N) * dt, 1.0, 1.0 / 12.0)[:, None]
    return sim, Problem(sim, src, sens, mode=mode, checkpoints=checkpoints), c, signal


def _loss(c, signal, problem, observed):
    from cuwave_b200.autograd import wave_traces

    traces = wave_traces(c, signal, problem)
    return 0.5 * ((traces - observed) ** 2).sum()


@pytest.mark.parametrize("mode,checkpoints", [("history", None), ("reconstruction", None),
                                              ("reconstruction", 2)])
def test_speed_gradient_matches_finite_differences(mode, checkpoints):
    sim, problem, c0, signal = _problem(mode, checkpoints)
    dev = torch.device("cuda")
    sig = torch.tensor(signal, device=dev)
    observed = torch.zeros((sim.N, 6), dtype=torch.float64, device=dev)
    # observed traces from a perturbed model, so the residual is not small
    c_obs = torch.tensor(c0 * 1.03, device=dev)
    from cuwave_b200.autograd import wave_traces

    observed = wave_traces(c_obs, sig, problem).detach()
    c = torch.tensor(c0, device=dev, requires_grad=True)
    loss = _loss(c, sig, problem, observed)
    loss.backward()
    grad = c.grad.cpu().numpy()
    # 16 random cells among those the misfit is sensitive to (a central difference at a
    # cell of near-zero gradient measures only the loss's round-off, eps * loss / h)
    lo = problem.sim.pml.width + 2
    inner = np.zeros(grad.shape, bool)
    inner[tuple(slice(lo, n - lo) for n in sim.Nx)] = True
    scale = np.abs(grad[inner]).max()
    candidates = np.argwhere(inner & (np.abs(grad) >= 0.05 * scale))
    rng = np.random.default_rng(7)
    cells = [tuple(candidates[i]) for i in rng.choice(len(candidates), 16, replace=False)]
    for cell in cells:
        h = 1e-5 * c0[cell]
        cp = c0.copy()
        cp[cell] += h
        cm = c0.copy()
        cm[cell] -= h
        lp = float(_loss(torch.tensor(cp, device=dev), sig, problem, observed))
        lm = float(_loss(torch.tensor(cm, device=dev), sig, problem, observed))
        fd = (lp - lm) / (2 * h)
        assert abs(grad[cell] - fd) <= 1e-5 * abs(fd) + 1e-7 * scale, (cell, grad[cell], fd)


def test_signal_gradient_matches_finite_differences():
    sim, problem, c0, signal = _problem("history")
    dev = torch.device("cuda")
    c = torch.tensor(c0, device=dev)
    observed = torch.zeros((sim.N, 6), dtype=torch.float64, device=dev)
    sig = torch.tensor(signal, device=dev, requires_grad=True)
    loss = _loss(c, sig, problem, observed)
    loss.backward()
    grad = sig.grad.cpu().numpy()
    scale = np.abs(grad).max()
    h = 1e-5 * np.abs(signal).max()
    for t in (5, 17, 33, 60):
        sp = signal.copy()
        sp[t, 0] += h
        sm = signal.copy()
        sm[t, 0] -= h
        lp = float(_loss(c, torch.tensor(sp, device=dev), problem, observed))
        lm = float(_loss(c, torch.tensor(sm, device=dev), problem, observed))
        fd = (lp - lm) / (2 * h)
        assert abs(grad[t, 0] - fd) <= 1e-6 * abs(fd) + 1e-8 * scale, (t, grad[t, 0], fd)


@pytest.mark.parametrize("ndim", [2, 3])
def test_reconstruction_mode_matches_history_mode(ndim):
    """Both memory modes differentiate the same discretisation: equal where the strip
    shields the rebuilt field, i.e. outside the PML layer and its reach."""
    sims = [_problem(m, ndim=ndim) for m in ("history", "reconstruction")]
    dev = torch.device("cuda")
    grads = []
    for sim, problem, c0, signal in sims:
        c = torch.tensor(c0, device=dev, requires_grad=True)
        sig = torch.tensor(signal, device=dev, requires_grad=True)
        observed = torch.zeros((sim.N, 6), dtype=torch.float64, device=dev)
        _loss(c, sig, problem, observed).backward()
        grads.append((c.grad.cpu().numpy(), sig.grad.cpu().numpy()))
    from cuwave_b200.sensitivity import reconstruction_nodes

    _, valid = reconstruction_nodes(sims[0][0], None)
    valid = valid.cpu().numpy()
    a, b = grads[0][0][valid], grads[1][0][valid]
    assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(a)
    np.testing.assert_allclose(grads[1][1], grads[0][1], rtol=1e-9, atol=1e-15)
