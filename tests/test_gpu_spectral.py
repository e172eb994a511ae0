"""spectral_sensitivity through the CUDA path (CWB_OP_DFT, CWB_OP_GRADIENT).

Bit for bit with the reference's own run on the spec*.npz fixtures under a cost linear
in the record (its derivative an input), to 1e-4 under `intensity` (whose transform is a
float32 matrix product, rounded differently by the two BLAS), and the properties
cuwave's SpectralTest pins (tests/sensitivity_test.py:1148-1203): agreement with the
exact adjoint on a damped domain once the runs decay, a region that keeps the gradient
inside it, the warning for a run that has not decayed, and the refusal of a cost off
the spectrum.
"""

import warnings
from dataclasses import replace

import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu

SPECTRAL = sorted(p.stem for p in cases.GOLDEN.glob("spec*.npz"))


def _fixture_run(fx, objective):
    from cuwave_b200 import Source
    from cuwave_b200.sensitivity import spectral_sensitivity

    sim, design = cases.product_sim(fx)
    source = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    region = fx["region"] if fx["region"].size else None
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        return spectral_sensitivity(sim, source, design.copy(), fx["sensors"],
                                    objective(sim), fx["frequencies"], region)


@pytest.mark.parametrize("name", SPECTRAL)
def test_spectral_matches_reference(name):
    fx = cases.load(name)
    coef = torch.as_tensor(fx["coef"], device="cuda")

    def linear(sim):
        def objective(traces):
            return float(torch.sum(coef * traces)), coef.clone()

        return objective

    cost, grads, traces, info = _fixture_run(fx, linear)
    np.testing.assert_array_equal(traces.cpu().numpy(), fx["traces"])
    np.testing.assert_array_equal(grads["mass"].cpu().numpy(), fx["g_mass"])
    np.testing.assert_array_equal(grads["stiff"].cpu().numpy(), fx["g_stiff"])
    assert cost == pytest.approx(float(fx["cost"]), rel=1e-5)
    assert info["decay"] == pytest.approx(float(fx["decay"]), rel=1e-6)
    assert info["fit"] == pytest.approx(float(fx["fit"]), rel=1e-3, abs=1e-12)


@pytest.mark.parametrize("name", SPECTRAL)
def test_spectral_intensity_matches_reference(name):
    from cuwave_b200.utils import intensity

    fx = cases.load(name)
    cost, grads, traces, info = _fixture_run(fx, lambda sim: intensity(sim, fx["frequencies"]))
    np.testing.assert_array_equal(traces.cpu().numpy(), fx["i_traces"])
    assert cost == pytest.approx(float(fx["i_cost"]), rel=1e-5)
    for key in ("mass", "stiff"):
        got, want = grads[key].cpu().numpy().astype(np.float64), fx[f"i_g_{key}"]
        assert cases.rel_l2(got, want) < 1e-4, key
    assert info["decay"] == pytest.approx(float(fx["i_decay"]), rel=1e-4)


def _problem(steps=900, beta=0.02, order=2):
    """cuwave's spectral problem: the float64 unit-square ScalarWave (30 x 28 nodes) of
    tests/sensitivity_test.py:122-135, 236-250, damped uniformly to `beta` (179-183)."""
    import math

    from cuwave_b200 import ScalarWave, Source, grid_coords, ricker, stable_dt

    res = 30
    Nx, dx = (res, res - 2), (1.0 / (res - 3),) * 2
    sim = ScalarWave(Nx=Nx, dx=dx, N=steps, dt=0.85 * stable_dt(dx, 1.0, order),
                     precision="float64", space_order=order, wavespeed=1.0, density=1.3)
    t = np.linspace(0, (steps - 1) * sim.dt, steps)
    signal = ricker(t, 1.0, 5.0) / np.prod(dx)
    source = Source(np.array([[1], [Nx[1] // 2]], np.int32), signal[:, None])
    sensors = np.array([[1, Nx[0] - 2, Nx[0] // 3], [5, Nx[1] - 2, Nx[1] // 3]], np.int32)
    x, y = grid_coords(sim.Nx, sim.dx)
    indicator = (1.0 + 0.25 * torch.sin(2 * math.pi * x) * torch.cos(3 * math.pi * y)).contiguous()
    minv = sim.inverse_inertia(indicator.clone())
    sim = replace(sim, damping=(2.0 * beta / sim.dt / minv).contiguous())
    return sim, source, sensors, indicator


FREQUENCIES = (5.0, 7.0)


def _both(steps=900, beta=0.02, region=None, order=2):
    from cuwave_b200.sensitivity import sensitivity, spectral_sensitivity
    from cuwave_b200.utils import intensity

    sim, source, sensors, indicator = _problem(steps, beta, order)
    objective = intensity(sim, FREQUENCIES)
    reference = sensitivity(sim, source, indicator.clone(), sensors, objective)
    spectral = spectral_sensitivity(sim, source, indicator.clone(), sensors, objective,
                                    FREQUENCIES, region)
    return sim, indicator, reference, spectral


@pytest.mark.parametrize("order", [2, 4])
def test_it_matches_sensitivity_once_the_fields_decay(order):
    from cuwave_b200.utils import _reparametrize

    sim, indicator, (c0, g0, _, _), (c1, g1, _, info) = _both(order=order)
    assert c0 == pytest.approx(c1, rel=1e-12)
    a, b = _reparametrize(sim, indicator, g1), _reparametrize(sim, indicator, g0)
    rel = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    assert info["decay"] < 1e-5
    assert rel < 1e-5, rel


def test_a_region_keeps_the_gradient_inside_it():
    from cuwave_b200.utils import _reparametrize

    sim, indicator, _, (_, whole, _, _) = _both()
    region = torch.zeros(sim.Nx_padded, dtype=torch.bool, device="cuda")
    region[10:20, 8:16] = True
    _, _, _, (_, part, _, _) = _both(region=region)
    a, b = _reparametrize(sim, indicator, part), _reparametrize(sim, indicator, whole)
    rel = float(torch.linalg.vector_norm(a[region] - b[region]) / torch.linalg.vector_norm(b[region]))
    assert rel < 1e-12, rel
    assert float(a[~region].abs().max()) == 0.0


def test_a_run_that_has_not_decayed_warns():
    with pytest.warns(RuntimeWarning, match="last period"):
        _both(steps=300, beta=0.002)


def test_a_cost_off_the_spectrum_is_refused():
    from cuwave_b200.sensitivity import l2_misfit, spectral_sensitivity

    sim, source, sensors, indicator = _problem(steps=600)
    objective = l2_misfit(np.zeros((sim.N, sensors.shape[1])))
    with pytest.raises(ValueError):
        spectral_sensitivity(sim, source, indicator, sensors, objective, FREQUENCIES)
