"""superposition_sensitivity through the CUDA path (CWB_OP_SUPERPOSED, CWB_OP_FRECHET).

Bit for bit with the reference's own run on the sup*.npz fixtures, and the properties
cuwave's SuperpositionTest pins (tests/sensitivity_test.py:770-907): the cost and
traces of `sensitivity` exactly, a gradient whose direction agrees with the exact
adjoint's, the warning past the usable cancellation, and the refusals.
"""

import warnings
from dataclasses import replace

import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu

SUPERPOSITION = sorted(p.stem for p in cases.GOLDEN.glob("sup*.npz"))


def _run(fx, scale=None, sim=None):
    from cuwave_b200 import Source
    from cuwave_b200.sensitivity import l2_misfit, superposition_sensitivity

    base, design = cases.product_sim(fx)
    sim = base if sim is None else sim
    source = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    scale = float(fx["scale"]) if scale is None else scale
    return superposition_sensitivity(sim, source, design.copy(), fx["sensors"],
                                     l2_misfit(fx["observed"]), scale=scale)


@pytest.mark.parametrize("name", SUPERPOSITION)
def test_superposition_matches_reference(name):
    fx = cases.load(name)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        cost, grads, traces, info = _run(fx)
    np.testing.assert_array_equal(traces.cpu().numpy(), fx["traces"])
    np.testing.assert_array_equal(grads["mass"].cpu().numpy(), fx["g_mass"])
    np.testing.assert_array_equal(grads["stiff"].cpu().numpy(), fx["g_stiff"])
    assert cost == pytest.approx(float(fx["cost"]), rel=1e-5)
    assert info["cancellation"] == pytest.approx(float(fx["cancellation"]), rel=1e-3)
    assert info["scale"] == float(fx["scale"])


def test_round_off_scale_warns():
    fx = cases.load("sup2d_r2_mixed")  # k = 0.01 leaves a cancellation past 1e5
    with pytest.warns(RuntimeWarning, match="cancellation"):
        _run(fx)


def _problem(N=150, res=40, density=1.3):
    """cuwave's superposition problem (tests/sensitivity_test.py:122-135, 156-162,
    236-250): a float64 ScalarWave of order 2 on the unit square, a Ricker source on a
    wall, sensors on a wall, a corner and inside, a smooth material and the energy
    reaching the sensors as the cost."""
    import math

    from cuwave_b200 import ScalarWave, Source, grid_coords, ricker, stable_dt
    from cuwave_b200.sensitivity import l2_misfit

    Nx, dx = (res, res - 2), (1.0 / (res - 3),) * 2
    sim = ScalarWave(Nx=Nx, dx=dx, N=N, dt=0.85 * stable_dt(dx, 1.0, 2), precision="float64",
                     space_order=2, wavespeed=1.0, density=density)
    t = np.linspace(0, (N - 1) * sim.dt, N)
    signal = ricker(t, 1.0, 5.0) / np.prod(dx)
    source = Source(np.array([[1], [Nx[1] // 2]], np.int32), signal[:, None])
    sensors = np.array([[1, Nx[0] - 2, Nx[0] // 3], [5, Nx[1] - 2, Nx[1] // 3]], np.int32)
    x, y = grid_coords(sim.Nx, sim.dx)
    indicator = (1.0 + 0.25 * torch.sin(2 * math.pi * x) * torch.cos(3 * math.pi * y)).contiguous()
    objective = l2_misfit(np.zeros((N, sensors.shape[1])))
    return sim, source, sensors, indicator, objective


def _discrepancy(sim, a, b):
    """Relative difference and cosine over the interior two nodes in from the walls."""
    sl = tuple(slice(2, n - 2) for n in sim.Nx)
    a, b = a[sl].double(), b[sl].double()
    rel = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    cos = float((a * b).sum() / (torch.linalg.vector_norm(a) * torch.linalg.vector_norm(b)))
    return rel, cos


def test_cost_and_traces_are_those_of_sensitivity_and_the_direction_agrees():
    from cuwave_b200.sensitivity import sensitivity, superposition_sensitivity
    from cuwave_b200.utils import _reparametrize

    sim, source, sensors, indicator, objective = _problem()
    c0, g0, t0, _ = sensitivity(sim, source, indicator.clone(), sensors, objective)
    c1, g1, t1, _ = superposition_sensitivity(sim, source, indicator.clone(), sensors, objective)
    # the same forward march: equal traces; the stored-history record is column-major
    # (as numpy gathers it), so the cost's float sum runs in another order
    assert torch.equal(t0, t1)
    assert c0 == pytest.approx(c1, rel=1e-12)
    # a different discretisation of the same derivative: the directions agree
    rel, cos = _discrepancy(sim, _reparametrize(sim, indicator, g1),
                            _reparametrize(sim, indicator, g0))
    assert rel < 0.25, rel
    assert cos > 0.98, cos


def test_cancellation_tracks_the_scale():
    from cuwave_b200.sensitivity import superposition_sensitivity

    sim, source, sensors, indicator, objective = _problem()
    loose = superposition_sensitivity(sim, source, indicator.clone(), sensors, objective,
                                      scale=1.0)[3]["cancellation"]
    tight = superposition_sensitivity(sim, source, indicator.clone(), sensors, objective,
                                      scale=1e-2)[3]["cancellation"]
    assert tight / loose == pytest.approx(100.0, abs=1.0)


def test_a_sensor_on_the_source_still_gives_the_right_gradient():
    from cuwave_b200.sensitivity import l2_misfit, sensitivity, superposition_sensitivity
    from cuwave_b200.utils import _reparametrize

    sim, source, sensors, indicator, _ = _problem()
    shared = np.concatenate((np.asarray(source.position), sensors[:, 2:]), axis=1)
    objective = l2_misfit(np.zeros((sim.N, shared.shape[1])))
    _, g1, _, _ = superposition_sensitivity(sim, source, indicator.clone(), shared, objective)
    _, g0, _, _ = sensitivity(sim, source, indicator.clone(), shared, objective)
    rel, cos = _discrepancy(sim, _reparametrize(sim, indicator, g1),
                            _reparametrize(sim, indicator, g0))
    assert rel < 0.25, rel
    assert cos > 0.98, cos


def test_lossy_steps_and_ghost_sensors_are_refused():
    from cuwave_b200 import Pml, Source
    from cuwave_b200.sensitivity import l2_misfit, superposition_sensitivity

    fx = cases.load("sup2d_r4")
    sim, design = cases.product_sim(fx)
    source = Source(fx["source"], fx["signal"])
    objective = l2_misfit(fx["observed"])
    with pytest.raises(NotImplementedError):
        superposition_sensitivity(replace(sim, pml=Pml(width=5, wavespeed=1.3)), source,
                                  design.copy(), fx["sensors"], objective)
    with pytest.raises(NotImplementedError):
        superposition_sensitivity(replace(sim, damping=np.zeros(sim.Nx_padded, np.float32)),
                                  source, design.copy(), fx["sensors"], objective)
    ghost = np.array([[sim.Nx[0] - 1], [5]], np.int32)
    with pytest.raises(ValueError):
        superposition_sensitivity(sim, source, design.copy(), ghost,
                                  l2_misfit(np.zeros((sim.N, 1), np.float32)))
