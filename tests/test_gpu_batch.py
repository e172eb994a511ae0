"""`simulate_batch`: many 2D problems of uneven size, order, length and boundaries stepped
together by the native batch (cwb_batch_*), against `simulate` on each, bit for bit."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(rng, Nx, order, N, *, pml=0, dirichlet=False, damping=False, nsens=5):
    from cuwave_b200 import AcousticWave, Dirichlet, Neumann, Pml, Source, ricker, sponge, stable_dt

    dx = (1.0, 1.0)
    c = 1.0 + 0.3 * rng.random((Nx[0], (Nx[1] + 31) // 32 * 32))
    dt = 0.5 * stable_dt(dx, float(c.max()), order)
    boundary = ((Dirichlet, Neumann), (Neumann, Dirichlet)) if dirichlet else Neumann
    sim = AcousticWave(Nx=Nx, dx=dx, N=N, dt=dt, space_order=order, boundary=boundary,
                       pml=Pml(width=pml, wavespeed=float(c.max())) if pml else None,
                       rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=0.5)
    indicator = AcousticWave.indicator_for_speed(c, 0.5)
    if damping:
        from dataclasses import replace

        sim = replace(sim, damping=sponge(sim, np.ones_like(indicator), 6, 0.1))
    t = np.arange(N) * dt
    signal = ricker(t, 1.0, 0.05)[:, None]
    position = np.array([[Nx[0] // 2], [Nx[1] // 3]], np.int32)
    sensors = np.stack([rng.integers(2, n - 2, nsens) for n in Nx]).astype(np.int32)
    return sim, Source(position, signal), indicator.astype(np.float32), sensors


def test_a_batch_of_uneven_problems_is_each_simulate():
    from cuwave_b200 import simulate
    from cuwave_b200.batch import simulate_batch

    rng = np.random.default_rng(5)
    specs = [
        dict(Nx=(64, 70), order=2, N=90),
        dict(Nx=(150, 133), order=4, N=120, pml=8),
        dict(Nx=(97, 201), order=8, N=75, dirichlet=True),
        dict(Nx=(80, 64), order=10, N=110, damping=True),
        dict(Nx=(121, 90), order=12, N=60, pml=10, dirichlet=True),
        dict(Nx=(70, 77), order=16, N=100),
        dict(Nx=(256, 300), order=6, N=130),
        dict(Nx=(64, 70), order=4, N=90),
    ]
    problems = [_problem(rng, **spec) for spec in specs]
    sims, sources, indicators, sensors = (list(x) for x in zip(*problems))
    batched = simulate_batch(sims, sources, [i.copy() for i in indicators], sensors)
    for k, (sim, source, indicator, sens) in enumerate(problems):
        field, traces = simulate(sim, source, indicator.copy(), sens)
        got_field, got_traces = batched[k]
        assert torch.equal(got_field, field), k
        assert torch.equal(got_traces, traces), k


def test_a_batch_matches_the_oracle():
    """The batch against the CPU oracle's restatement of the reference's step sequence,
    not only against `simulate`: problems of four radius groups (orders 2, 6, 8 and 16),
    Neumann and mixed Dirichlet faces, different lengths, fields and traces to the bit."""
    from oracle import oracle as o

    from cuwave_b200.batch import simulate_batch

    rng = np.random.default_rng(11)
    specs = [dict(Nx=(64, 70), order=2, N=40), dict(Nx=(97, 201), order=8, N=30, dirichlet=True),
             dict(Nx=(70, 77), order=16, N=35), dict(Nx=(150, 130), order=6, N=25)]
    problems = [_problem(rng, **spec) for spec in specs]
    sims, sources, indicators, sensors = (list(x) for x in zip(*problems))
    batched = simulate_batch(sims, sources, [i.copy() for i in indicators], sensors)
    for k, (sim, source, indicator, sens) in enumerate(problems):
        Nx = sim.Nx
        R = sim.space_order // 2
        stiff, minv = o.acoustic_materials(Nx, indicator.copy(), 1.0, 1.0, 1.0, 0.5, np.float32)
        shape = sim.Nx_padded
        flat = lambda q: (q[0].astype(np.int64) * shape[1] + q[1]).astype(np.int32)  # noqa: E731
        dirichlet = 0b1001 if specs[k].get("dirichlet") else 0
        case = o.Case(Nx=Nx, R=R, coeffs=o.cell_coefficients(R, "optimized"),
                      factors=[np.float32(2.0 * sim.dt**2)] * 2, dt=sim.dt, stiff=stiff, minv=minv,
                      dtype=np.float32, dirichlet=dirichlet,
                      source_lin=flat(np.asarray(source.position)),
                      signal=np.asarray(source.signal, np.float32), sensor_lin=flat(sens))
        case.source_weight = case.excitation_weights(case.source_lin)
        field, traces = case.forward(sim.N)
        got_field, got_traces = batched[k]
        np.testing.assert_array_equal(got_traces.cpu().numpy(), traces)
        np.testing.assert_array_equal(got_field.cpu().numpy(), field[:, : Nx[1]])


def test_the_batch_refuses_what_it_does_not_step():
    from cuwave_b200 import AcousticWave
    from cuwave_b200.batch import simulate_batch

    rng = np.random.default_rng(1)
    sim, source, indicator, sensors = _problem(rng, (64, 70), 4, 20)
    # a density that varies: the stiffness is not uniform
    varied = AcousticWave(Nx=sim.Nx, dx=sim.dx, N=sim.N, dt=sim.dt, space_order=4, rho1=1.0,
                          rho2=2.0, kappa1=1.0, kappa2=0.5)
    with pytest.raises(NotImplementedError):
        simulate_batch([varied], [source], [rng.random(sim.Nx_padded).astype(np.float32)])
    sim3 = AcousticWave(Nx=(20, 20, 20), dx=(1.0, 1.0, 1.0), N=5, dt=0.1, space_order=2,
                        rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=0.5)
    with pytest.raises(NotImplementedError):
        simulate_batch([sim3], [source], [np.zeros(sim3.Nx_padded, np.float32)])
