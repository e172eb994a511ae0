"""Masked domains (`domain`, `dirichlet`) through the CUDA path.

Bit for bit with the reference's own run on the mask*.npz fixtures (a disk, an obstacle
held at zero inside it, a held row; 2D and 3D; orders 2 to 12): the forward field and
traces, and the signal gradient stepped back by the graded step. And the properties
cuwave's DomainTest pins (tests/wave_test.py:186-320): the material outside the domain is
never read, a domain covering everything is the plain scheme, a held row is the method
of images, the graded operator is its own adjoint at order 2, and the refusals.
"""

from dataclasses import replace

import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu

MASKED = sorted(p.stem for p in cases.GOLDEN.glob("mask*.npz"))


def _masked_sim(fx):
    sim, design = cases.product_sim(fx)
    domain = fx["domain"] if fx["domain"].size else None
    dirichlet = fx["dirichlet_mask"] if fx["dirichlet_mask"].size else None
    return replace(sim, domain=domain, dirichlet=dirichlet), design


@pytest.mark.parametrize("name", MASKED)
def test_masked_domain_matches_reference(name):
    from cuwave_b200 import Source, simulate
    from cuwave_b200.sensitivity import l2_misfit, source_sensitivity
    from cuwave_b200.wave import domain_cells

    fx = cases.load(name)
    sim, design = _masked_sim(fx)
    Nx = sim.Nx
    interior = tuple(slice(1, n - 1) for n in Nx)
    np.testing.assert_array_equal(domain_cells(sim).cpu().numpy()[interior], fx["cells"][interior])
    source = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
    field, traces = simulate(sim, source, design.copy(), fx["sensors"])
    np.testing.assert_array_equal(field.cpu().numpy(), fx["field"])
    np.testing.assert_array_equal(traces.cpu().numpy(), fx["traces"])
    cost, gradient, _, _ = source_sensitivity(sim, source, design.copy(), fx["sensors"],
                                              l2_misfit(fx["observed"]))
    np.testing.assert_array_equal(gradient.cpu().numpy(), fx["source_gradient"])
    assert cost == pytest.approx(float(fx["source_cost"]), rel=1e-5)


def _disk(precision="float32", order=4, N=100):
    """A ScalarWave on the unit square stepped inside a disk (tests/wave_test.py:52-86)."""
    from cuwave_b200 import ScalarWave, Source, grid_coords, stable_dt

    Nx = (40, 48)
    dx = tuple(1.0 / (n - 3) for n in Nx)
    sim = ScalarWave(Nx=Nx, dx=dx, N=N, dt=0.5 * stable_dt(dx, 1.0, 4), space_order=order,
                     precision=precision, wavespeed=1.0, density=1.0)
    uniform = np.random.RandomState(0).rand(*sim.Nx_padded)
    indicator = (1.0 + 0.2 * uniform).astype(sim.np_dtype)
    signal = np.sin(0.3 * np.arange(N))[:, None]
    source = Source(np.array([[20], [24]], np.int32), signal.astype(sim.np_dtype))
    X = grid_coords(sim.Nx, sim.dx)
    domain = ((X[0] - 0.5) ** 2 + (X[1] - 0.5) ** 2 <= 0.42**2).cpu().numpy()
    sensors = np.array([[12, 20, 28, 7], [14, 36, 20, 24]], np.int32)
    return replace(sim, domain=domain), source, indicator, sensors


def test_the_material_outside_is_never_read():
    from cuwave_b200 import simulate

    sim, source, indicator, sensors = _disk()
    voided = np.where(sim.domain, indicator, sim.np_dtype(1e-4))
    filled = np.where(sim.domain, indicator, sim.np_dtype(1.0))
    for a, b in zip(simulate(sim, source, voided, sensors), simulate(sim, source, filled, sensors)):
        assert torch.equal(a, b)


def test_a_domain_covering_everything_is_the_plain_scheme():
    from cuwave_b200 import simulate

    sim, source, indicator, sensors = _disk()
    plain = simulate(replace(sim, domain=None), source, indicator, sensors)
    covered = simulate(replace(sim, domain=np.ones(sim.Nx_padded, bool)), source, indicator,
                       sensors)
    # every node deep, so the same arithmetic as the unmasked step
    for a, b in zip(plain, covered):
        assert torch.equal(a, b)


def test_a_held_row_is_the_method_of_images():
    from cuwave_b200 import ScalarWave, Source, simulate, stable_dt

    dx = (0.02, 0.02)
    sim = ScalarWave(Nx=(40, 36), dx=dx, N=150, dt=0.9 * stable_dt(dx, 1.0), precision="float64",
                     wavespeed=1.0, density=1.0)
    signal = np.sin(0.3 * np.arange(sim.N))
    one = Source(np.array([[12], [15]], np.int32), signal[:, None])
    pair = Source(np.array([[12, 27], [15, 15]], np.int32), np.stack([signal, -signal], 1))
    indicator = np.ones(sim.Nx_padded)
    imaged = simulate(sim, pair, indicator)
    held_row = np.zeros(sim.Nx_padded, bool)
    held_row[20] = True
    held = simulate(replace(sim, dirichlet=held_row), one, indicator)
    below = (slice(1, 20), slice(1, 35))
    scale = float(imaged[below].abs().max())
    assert float((held[below] - imaged[below]).abs().max()) <= 1e-12 * scale


def test_the_graded_operator_is_its_own_adjoint():
    from cuwave_b200 import Source, simulate
    from cuwave_b200.sensitivity import l2_misfit, source_sensitivity

    sim, source, indicator, sensors = _disk("float64", order=2)
    objective = l2_misfit(np.zeros((sim.N, sensors.shape[1])))
    gradient = source_sensitivity(sim, source, indicator, sensors, objective)[1]
    direction = torch.as_tensor(np.random.RandomState(1).standard_normal(source.signal.shape),
                                device="cuda")
    signal = torch.as_tensor(source.signal, device="cuda")
    h = 1e-3

    def cost(s):
        return objective(simulate(sim, Source(source.position, s), indicator, sensors)[1])[0]

    reference = (cost(signal + h * direction) - cost(signal - h * direction)) / (2 * h)
    assert float((gradient * direction).sum()) / reference == pytest.approx(1.0, abs=1e-8)


def test_points_off_the_stepped_nodes_and_gradients_are_refused():
    from cuwave_b200 import simulate
    from cuwave_b200.sensitivity import l2_misfit, sensitivity

    sim, source, indicator, sensors = _disk()
    with pytest.raises(ValueError):
        simulate(sim, source, indicator, np.array([[2], [2]], np.int32))
    plain = replace(sim, domain=None)
    held = np.zeros(sim.Nx_padded, bool)
    held[20, 24] = True
    with pytest.raises(ValueError):
        simulate(replace(plain, dirichlet=held), source, indicator, sensors)
    with pytest.raises(ValueError):
        simulate(replace(plain, domain=np.zeros(sim.Nx_padded, bool)), source, indicator, sensors)
    with pytest.raises(NotImplementedError):
        sensitivity(sim, source, indicator, sensors, l2_misfit(np.zeros((sim.N, 4))))
