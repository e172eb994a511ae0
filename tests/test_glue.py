"""The shot glue's host arithmetic and the oracle on off-node shots, against the reference.

The fixtures distribute*.npz and glue*.npz come from cuwave's own utils.py run by
make_golden.py: the corner nodes and weights of coordinates between nodes, the source
columns and their transpose, and whole multi-shot misfit gradients.
"""

import numpy as np
import pytest
import torch

import cases
from oracle import oracle as o

DISTRIBUTE = sorted(p.stem for p in cases.GOLDEN.glob("distribute*.npz"))
GLUE = sorted(p.stem for p in cases.GOLDEN.glob("glue*.npz"))


def _grid_sim(fx):
    from cuwave_b200 import AcousticWave

    Nx = tuple(int(n) for n in fx["Nx"])
    return AcousticWave(
        Nx=Nx, dx=tuple(float(d) for d in fx["dx"]), N=7, dt=0.1,
        precision=str(fx["precision"]), space_order=4, rho1=1.0, rho2=1.0, kappa1=1.0,
        kappa2=0.5,
    )


@pytest.mark.parametrize("name", DISTRIBUTE)
def test_cell_corners_match_reference(name):
    from cuwave_b200.utils import cell_corners

    fx = cases.load(name)
    sim = _grid_sim(fx)
    dtype = cases.dtype_of(fx)
    nodes, weights = cell_corners(sim, fx["coords"])
    np.testing.assert_array_equal(nodes, fx["nodes"])
    np.testing.assert_array_equal(weights.astype(dtype), fx["weights"])
    nodes, weights = cell_corners(sim, fx["coords"], direction=[[-1.5]])
    np.testing.assert_array_equal(nodes, fx["scaled_nodes"])
    np.testing.assert_array_equal(weights.astype(dtype), fx["scaled_weights"])


@pytest.mark.parametrize("name", DISTRIBUTE)
def test_source_columns_match_reference(name):
    from cuwave_b200.utils import cell_corners, gather_columns, spread_columns

    fx = cases.load(name)
    sim = _grid_sim(fx)
    _, weights = cell_corners(sim, fx["coords"])
    w = torch.as_tensor(weights).to(sim.dtype)
    volume = float(np.prod(sim.dx))
    signal = torch.as_tensor(fx["signal"]).to(sim.dtype)
    np.testing.assert_array_equal(spread_columns(signal, w, volume).numpy(), fx["columns_out"])
    columns = torch.as_tensor(fx["columns_in"])
    np.testing.assert_array_equal(gather_columns(columns, w, volume).numpy(), fx["collected"])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_corner_sum_follows_numpy(dtype):
    from cuwave_b200.utils import corner_sum

    rng = np.random.default_rng(7)
    for n in list(range(1, 20)) + [32, 37]:
        x = (rng.standard_normal((50, 9, n)) * np.exp(rng.uniform(-25, 25, (50, 9, n)))).astype(dtype)
        np.testing.assert_array_equal(corner_sum(torch.as_tensor(x)).numpy(), x.sum(-1))
        # a column-major table: numpy adds the strided corners one after another
        table = np.asfortranarray(x.reshape(50, -1))
        want = (table.reshape(50, 9, n) * np.ones(n, dtype)).sum(2)
        got = corner_sum(torch.as_tensor(x) * torch.ones(n, dtype=torch.as_tensor(x).dtype),
                         pairwise=False)
        np.testing.assert_array_equal(got.numpy(), want)


def test_coordinates_outside_the_domain_raise():
    from cuwave_b200.utils import cell_corners

    sim = _grid_sim(cases.load("distribute2d"))
    length = (sim.Nx[0] - 3) * sim.dx[0]
    cell_corners(sim, [[length * (1 + 1e-9), 1.0]])
    with pytest.raises(ValueError):
        cell_corners(sim, [[length + 0.01, 1.0]])
    with pytest.raises(ValueError):
        cell_corners(sim, [[1.0, -0.01]])
    with pytest.raises(ValueError):
        cell_corners(sim, [[1.0, 1.0, 1.0]])
    with pytest.raises(ValueError):
        cell_corners(sim, [[1.0, 1.0], [2.0, 2.0]], direction=[[1.0], [1.0], [1.0]])


def _lift(weights, objective, column_major=False):
    """The receiver objective on the node record, as Sensors.objective does it.

    The reference's stored-history sensitivity gathers its record column-major, and
    numpy then sums a cell's corners one after another instead of pairwise:
    `column_major` lays the oracle's record out the same way.
    """
    count = weights.shape[0]

    def wrapped(record):
        if column_major:
            record = np.asfortranarray(record)
        traces = (record.reshape(record.shape[0], count, -1) * weights).sum(2)
        cost, dphi = objective(traces)
        return cost, (dphi[:, :, None] * weights).reshape(dphi.shape[0], -1)

    return wrapped


def _jacobian(fx):
    if bool(fx["scalar"]):
        return 1.0, 1.0
    return 1 / float(fx["kappa2"]) - 1.0, 0.0


def _oracle_shot(fx, position, signal):
    case = cases.oracle_case(fx)
    case.source_lin = cases.flat(fx, position)
    case.signal = np.ascontiguousarray(signal)
    case.source_weight = case.excitation_weights(case.source_lin)
    case.sensor_lin = cases.flat(fx, fx["sensor_nodes"])
    return case


@pytest.mark.parametrize("name", GLUE)
def test_glue_host_and_oracle_match_reference(name):
    """Shot columns from the host glue, then the oracle's forward and adjoint per shot."""
    from cuwave_b200.utils import cell_corners, gather_columns, spread_columns

    fx = cases.load(name)
    sim, _ = cases.product_sim(fx)
    N = int(fx["N"])
    nodes, weights = cell_corners(sim, fx["receiver_coords"])
    np.testing.assert_array_equal(nodes, fx["sensor_nodes"])
    w = weights.astype(cases.dtype_of(fx))
    np.testing.assert_array_equal(w, fx["sensor_weights"])
    signal = torch.as_tensor(fx["signal"][:, 0]).to(sim.dtype)
    shots = []
    for k, coord in enumerate(fx["shot_coords"]):
        nodes, sw = cell_corners(sim, coord)
        np.testing.assert_array_equal(nodes, fx[f"shot{k}_position"])
        columns = spread_columns(signal[:, None], torch.as_tensor(sw).to(sim.dtype), 1.0)
        np.testing.assert_array_equal(columns.numpy(), fx[f"shot{k}_signal"])
        shots.append((nodes, columns.numpy()))

    # the stacked shot: one forward pass, traces through the corner weights
    case = _oracle_shot(fx, fx["stacked_position"], fx["stacked_signal"])
    _, record = case.forward(N)
    traces = (record.reshape(N, w.shape[0], -1) * w).sum(2)
    np.testing.assert_array_equal(traces, fx["stacked_traces"])

    # misfit_gradient: one adjoint per shot, reparametrized and summed in shot order
    d_mass, d_stiff = _jacobian(fx)
    gradient = np.zeros_like(fx["gradient"])
    total = 0.0
    for (position, columns), observed in zip(shots, fx["observed"]):
        case = _oracle_shot(fx, position, columns)
        cost, grads, _ = case.sensitivity(N, _lift(w, o.l2(observed), True))
        total += cost
        gradient += d_mass * grads["mass"] + d_stiff * grads["stiff"]
    np.testing.assert_array_equal(gradient, fx["gradient"])
    assert total == pytest.approx(float(fx["gradient_cost"]), rel=1e-5)

    # the energy of the stacked shot
    scale = float(np.prod(sim.dx)) * sim.dt

    def energy(traces):
        return 0.5 * scale * float(np.sum(traces**2)), scale * traces

    case = _oracle_shot(fx, fx["stacked_position"], fx["stacked_signal"])
    cost, grads, _ = case.sensitivity(N, _lift(w, energy, True))
    np.testing.assert_array_equal(d_mass * grads["mass"] + d_stiff * grads["stiff"],
                                  fx["energy_gradient"])
    assert cost == pytest.approx(float(fx["energy_cost"]), rel=1e-5)

    # the signal gradient of the first shot, collected back onto its coordinate
    position, columns = shots[0]
    case = _oracle_shot(fx, position, columns)
    _, node_gradient, _ = case.source_sensitivity(N, _lift(w, o.l2(fx["observed"][0])))
    np.testing.assert_array_equal(node_gradient, fx["source_columns"])
    _, sw = cell_corners(sim, fx["shot_coords"][:1])
    collected = gather_columns(torch.as_tensor(node_gradient), torch.as_tensor(sw).to(sim.dtype), 1.0)
    np.testing.assert_array_equal(collected.numpy(), fx["source_signal_gradient"])
