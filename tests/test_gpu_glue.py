"""The shot glue through the CUDA path against the reference's own run (glue*.npz).

Off-node shots and receivers, the traces of every shot, the misfit and its gradient
summed over the shots (stored history and reconstruction), a stacked shot's energy
gradient and the signal gradient collected back onto a coordinate: all bit for bit
with cuwave's utils.py on its host fallback, the costs (float sums) to 1e-5.
"""

import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu

GLUE = sorted(p.stem for p in cases.GOLDEN.glob("glue*.npz"))


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("name", GLUE)
def test_misfit_gradient_matches_reference(name):
    from cuwave_b200.sensitivity import l2_misfit, reconstruction_sensitivity, source_sensitivity
    from cuwave_b200.utils import (
        Sensors, collect_source, energy, measure, misfit, misfit_gradient, point_source,
        response_gradient, shots, stack,
    )

    fx = cases.load(name)
    sim, design = cases.product_sim(fx)
    dev = torch.device("cuda")

    def fresh():
        return torch.as_tensor(design, device=dev).clone()

    signal = fx["signal"][:, 0]
    sources = shots(sim, fx["shot_coords"], signal)
    for k, s in enumerate(sources):
        np.testing.assert_array_equal(_np(s.position), fx[f"shot{k}_position"])
        np.testing.assert_array_equal(_np(s.signal), fx[f"shot{k}_signal"])
    sensors = Sensors(sim, fx["receiver_coords"])
    np.testing.assert_array_equal(_np(sensors.nodes), fx["sensor_nodes"])
    np.testing.assert_array_equal(_np(sensors.weights), fx["sensor_weights"])

    perturbed = fresh() * 0.95
    observed = measure(sim, sources, perturbed, sensors, devices=(0,))
    np.testing.assert_array_equal(np.stack([_np(o) for o in observed]), fx["observed"])
    observed = [torch.as_tensor(o, device=dev) for o in fx["observed"]]

    cost = misfit(sim, sources, fresh(), sensors, observed)
    assert cost == pytest.approx(float(fx["misfit"]), rel=1e-5)
    gcost, gradient = misfit_gradient(sim, sources, fresh(), sensors, observed)
    np.testing.assert_array_equal(_np(gradient), fx["gradient"])
    assert gcost == pytest.approx(float(fx["gradient_cost"]), rel=1e-5)
    rcost, rgradient = misfit_gradient(sim, sources, fresh(), sensors, observed,
                                       adjoint=reconstruction_sensitivity)
    np.testing.assert_array_equal(_np(rgradient), fx["rec_gradient"])
    assert rcost == pytest.approx(float(fx["rec_cost"]), rel=1e-5)

    stacked = stack(sources)
    np.testing.assert_array_equal(_np(stacked.position), fx["stacked_position"])
    np.testing.assert_array_equal(_np(stacked.signal), fx["stacked_signal"])
    traces = measure(sim, [stacked], fresh(), sensors)[0]
    np.testing.assert_array_equal(_np(traces), fx["stacked_traces"])
    ecost, egradient = response_gradient(sim, stacked, fresh(), sensors.nodes,
                                         sensors.objective(energy(sim)))
    np.testing.assert_array_equal(_np(egradient), fx["energy_gradient"])
    assert ecost == pytest.approx(float(fx["energy_cost"]), rel=1e-5)

    one = point_source(sim, fx["shot_coords"][:1], signal)
    scost, columns, _, _ = source_sensitivity(sim, one, fresh(), sensors.nodes,
                                              sensors.objective(l2_misfit(observed[0])))
    np.testing.assert_array_equal(_np(columns), fx["source_columns"])
    collected = collect_source(sim, fx["shot_coords"][:1], columns)
    np.testing.assert_array_equal(_np(collected), fx["source_signal_gradient"])
    assert scost == pytest.approx(float(fx["source_cost"]), rel=1e-5)


def test_glue_arguments_are_checked():
    from cuwave_b200.utils import Sensors, measure, point_source

    fx = cases.load(GLUE[0])
    sim, design = cases.product_sim(fx)
    with pytest.raises(ValueError):
        point_source(sim, [[1.0, 2.0], [3.0, 4.0]], np.zeros((int(fx["N"]), 3)))
    with pytest.raises(ValueError):
        Sensors(sim, [[1000.0, 2.0]])
    with pytest.raises(NotImplementedError):
        measure(sim, [], design, Sensors(sim, [[3.0, 4.0]]), devices=(0, 1))


@pytest.mark.parametrize("name", GLUE)
def test_misfit_gradient_lanes_match_one_at_a_time(name):
    """Shots run side by side on their own streams and plans (`lanes`) give the gradient
    and cost of the shots run in turn, bit for bit, with either adjoint."""
    from cuwave_b200.sensitivity import reconstruction_sensitivity
    from cuwave_b200.utils import Sensors, misfit_gradient, shots

    fx = cases.load(name)
    sim, design = cases.product_sim(fx)
    dev = torch.device("cuda")
    signal = fx["signal"][:, 0]
    coords = np.concatenate([fx["shot_coords"]] * 3)  # more shots than lanes
    sources = shots(sim, coords, signal)
    sensors = Sensors(sim, fx["receiver_coords"])
    observed = [torch.as_tensor(fx["observed"][k % len(fx["observed"])], device=dev)
                for k in range(len(sources))]
    for adjoint in (None, reconstruction_sensitivity):
        kw = {} if adjoint is None else {"adjoint": adjoint}
        results = {}
        for lanes in (1, 3):
            ind = torch.as_tensor(design, device=dev).clone()
            results[lanes] = misfit_gradient(sim, sources, ind, sensors, observed, lanes=lanes, **kw)
        assert results[1][0] == results[3][0]
        np.testing.assert_array_equal(_np(results[1][1]), _np(results[3][1]))
    from cuwave_b200.utils import measure

    ind = torch.as_tensor(design, device=dev).clone()
    one = measure(sim, sources, ind, sensors, lanes=1)
    side = measure(sim, sources, ind, sensors, lanes=3)
    for a, b in zip(one, side):
        np.testing.assert_array_equal(_np(a), _np(b))
