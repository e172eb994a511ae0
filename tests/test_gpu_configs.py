"""Parity at the sizes of the benchmark workloads, not only on the small fixtures.

* The 2D forward job in full: a 512 x 512 grid, radius 4, 2000 steps, speed 1 plus eight
  seeded Gaussian blobs, a Ricker source at the centre, 64 receivers on row 51, Neumann
  faces. The CUDA path against the reference's own kernels compiled for the host
  (oracle/_ref, the reference's scalar.cu stepped in its `simulate` order): equal to the
  bit, field and traces. The float64 run of the same scheme on the same inputs gives
  the float32 error of both (stated in the assertion's bound: measured 4.0e-6 relative
  L2 on the traces, 5.6e-6 on the field).
* The 2D gradient job at its full grid: 2048 x 2048, radius 4, a 20-cell pml, 256
  receivers, 300 of its 3000 steps (the source and the receivers moved close together
  so the wave reaches them): `sensitivity` against the oracle's restatement of the
  reference's stored-history adjoint (cuwave sensitivity.py:384-497, pinned bit for bit
  to the reference's fixtures), `reconstruction_sensitivity` against it within 1e-4, and
  dL/dc in float64 against central differences on 16 cells.
"""

import os

import numpy as np
import pytest
import torch

import bench
import cases
from oracle import oracle as o

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _threads() -> int:
    return os.cpu_count() or 1


def test_full_2d_forward_job_matches_reference_kernels():
    from cuwave_b200 import Source, simulate

    w = bench.blob_workload(512, 2000)
    path, _ = o.ref_library(2, 4, "optimized", "float32")
    if not path.exists():
        pytest.skip(f"{path.name} not built")
    sim = bench.make_sim_2d(w)
    field, traces = simulate(sim, Source(w["source"], w["signal"]), w["indicator"].copy(), w["sensors"])
    field, traces = field.cpu().numpy(), traces.cpu().numpy()
    ref_field, ref_traces = o.ref_simulate(bench.reference_case(w, np.float32), w["steps"],
                                           threads=_threads())
    ref_field = ref_field[:, : w["Nx"][1]]
    assert np.abs(ref_traces).max() > 1e-3, "the wave must reach the receivers"
    assert cases.rel_l2(traces, ref_traces) <= TOL
    assert cases.rel_l2(field, ref_field) <= TOL
    np.testing.assert_array_equal(traces, ref_traces)
    np.testing.assert_array_equal(field, ref_field)
    # the float32 scheme (both builds, equal to the bit) against float64
    f64, t64 = o.ref_simulate(bench.reference_case(w, np.float64), w["steps"], threads=_threads())
    terr = cases.rel_l2(traces, t64)
    ferr = cases.rel_l2(field, f64[:, : w["Nx"][1]])
    print(f"float32 against float64: traces {terr:.2e}, field {ferr:.2e} relative L2")
    assert 0 < terr < 2e-5 and 0 < ferr < 2e-5, (terr, ferr)


@pytest.fixture(scope="module")
def gradient_job():
    from cuwave_b200 import Source, simulate

    w = bench.sensitivity_workload()
    sim = bench.make_sim_2d(w)
    source = Source(w["source"], w["signal"])
    _, observed = simulate(sim, source, w["indicator_obs"].copy(), w["sensors"])
    return w, sim, source, observed.cpu().numpy()


def test_gradient_job_matches_oracle(gradient_job):
    from cuwave_b200.sensitivity import l2_misfit, reconstruction_nodes, reconstruction_sensitivity, sensitivity

    w, sim, source, observed = gradient_job
    cost, grads, traces, _ = sensitivity(sim, source, w["indicator"].copy(), w["sensors"], l2_misfit(observed))
    case = bench.reference_case(w, np.float32)
    os.environ["OMP_NUM_THREADS"] = str(_threads())
    ref_cost, ref, ref_traces = case.sensitivity(w["steps"], o.l2(observed))
    n = w["Nx"][1]
    assert np.abs(ref_traces).max() > 1e-4 and ref_cost > 0, "the wave must reach the receivers"
    np.testing.assert_array_equal(traces.cpu().numpy(), ref_traces)
    for key in ("mass", "stiff"):
        got = grads[key].cpu().numpy()
        assert cases.rel_l2(got[:, :n], ref[key][:, :n]) <= 1e-4, key
        np.testing.assert_array_equal(got[:, :n], ref[key][:, :n])
    assert cost == pytest.approx(ref_cost, rel=1e-5)
    # memory independent of the steps: the strip replay, within 1e-4 where it reaches
    _, rec, _, info = reconstruction_sensitivity(sim, source, w["indicator"].copy(), w["sensors"],
                                                 l2_misfit(observed))
    _, valid = reconstruction_nodes(sim, torch.as_tensor(w["indicator"]))
    a = rec["mass"][valid].cpu().numpy()
    b = grads["mass"][valid].cpu().numpy()
    assert cases.rel_l2(a, b) <= 1e-4, cases.rel_l2(a, b)


def test_gradient_job_speed_gradient_matches_finite_differences(gradient_job):
    """dL/dc through the autograd Function in float64 against central differences on 16
    cells drawn among those whose gradient is at least 5% of the largest."""
    from cuwave_b200.autograd import Problem, wave_traces

    w, _, _, observed = gradient_job
    sim = bench.make_sim_2d(w, precision="float64")
    problem = Problem(sim, w["source"], w["sensors"], mode="history")
    dev = torch.device("cuda")
    n = w["Nx"][1]
    c0 = np.ones(sim.Nx_padded)
    c0[:, :n] = w["speed"]
    sig = torch.tensor(w["signal"], dtype=torch.float64, device=dev)
    obs = torch.tensor(observed, dtype=torch.float64, device=dev)

    def loss(c):
        return 0.5 * ((wave_traces(c, sig, problem) - obs) ** 2).sum()

    c = torch.tensor(c0, device=dev, requires_grad=True)
    loss(c).backward()
    grad = c.grad.cpu().numpy()
    lo = w["width"] + 2
    inner = np.zeros(grad.shape, bool)
    inner[lo:n - lo, lo:n - lo] = True
    scale = np.abs(grad[inner]).max()
    candidates = np.argwhere(inner & (np.abs(grad) >= 0.05 * scale))
    rng = np.random.default_rng(11)
    cells = [tuple(candidates[i]) for i in rng.choice(len(candidates), 16, replace=False)]
    for cell in cells:
        h = 1e-5 * c0[cell]
        cp, cm = c0.copy(), c0.copy()
        cp[cell] += h
        cm[cell] -= h
        with torch.no_grad():
            lp = float(loss(torch.tensor(cp, device=dev)))
            lm = float(loss(torch.tensor(cm, device=dev)))
        fd = (lp - lm) / (2 * h)
        assert abs(grad[cell] - fd) <= 1e-5 * abs(fd) + 1e-7 * scale, (cell, grad[cell], fd)
