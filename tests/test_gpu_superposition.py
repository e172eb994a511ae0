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


def test_cost_and_traces_are_those_of_sensitivity_and_the_direction_agrees():
    from cuwave_b200 import Source
    from cuwave_b200.sensitivity import l2_misfit, sensitivity

    fx = cases.load("sup2d_r4_f64")
    sim, design = cases.product_sim(fx)
    source = Source(fx["source"], fx["signal"])
    c0, g0, t0, _ = sensitivity(sim, source, design.copy(), fx["sensors"],
                                l2_misfit(fx["observed"]))
    c1, g1, t1, _ = _run(fx)
    assert c0 == c1
    assert torch.equal(t0, t1)
    # a different discretisation of the same derivative: the directions agree
    a = torch.cat([g1["mass"].flatten(), g1["stiff"].flatten()]).double()
    b = torch.cat([g0["mass"].flatten(), g0["stiff"].flatten()]).double()
    rel = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    cos = float(a @ b / (torch.linalg.vector_norm(a) * torch.linalg.vector_norm(b)))
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
