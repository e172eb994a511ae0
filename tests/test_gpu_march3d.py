"""All the steps of a small 3D grid in one cooperative launch (march3d_kernel, the role of
cuwave's 3D blocked_kernel on a grid that stays in L2) against the CPU oracle, and against
the per-step march, bit for bit: radius 1 to 8, heterogeneous and uniform stiffness, pml
slabs, Dirichlet and Neumann faces, damping, float64, sources and receivers, step counts
that split into several chunks of tiles."""

import os

import numpy as np
import pytest
import torch

import cases
from test_gpu_parity import _product, _random_case

pytestmark = pytest.mark.gpu


def _run(case, meta, mode):
    from cuwave_b200 import _native as nat

    os.environ["CWB_MARCH3D"] = mode
    try:
        n0 = nat.launches()
        field, traces = _product(case, meta)
        torch.cuda.synchronize()
        return field, traces, nat.launches() - n0
    finally:
        os.environ["CWB_MARCH3D"] = "0"


@pytest.mark.parametrize("R,kw", [
    (1, dict(uniform=True)),
    (2, dict(pml=4, dirichlet=0b100110)),
    (3, dict(uniform=True, pml=5, nsrc=6)),
    (4, dict(uniform=True, pml=6, dirichlet=0b011001, nsrc=6, nsens=9)),
    (4, dict(damping=True)),
    (5, dict(pml=3)),
    (8, dict(uniform=True, dirichlet=0b111111)),
    (3, dict(dtype=np.float64, pml=4)),
])
def test_march3d_matches_oracle_and_per_step(R, kw):
    case, meta = _random_case(3, R, seed=70 + R, Nx=(45, 37, 139), **kw)
    f_one, t_one, l_one = _run(case, meta, "2")
    f_step, t_step, l_step = _run(case, meta, "0")
    # the cooperative march launches twice (the counter, the march), the other every step
    assert l_one < l_step, (l_one, l_step)
    ref_field, ref_traces = case.forward(meta["N"])
    np.testing.assert_array_equal(t_one, ref_traces)
    np.testing.assert_array_equal(f_one, ref_field)
    np.testing.assert_array_equal(t_one, t_step)
    np.testing.assert_array_equal(f_one, f_step)


@pytest.mark.parametrize("name", [n for n in cases.FORWARD if n.startswith("fwd3d")])
def test_march3d_matches_reference_fixtures(name):
    """`simulate` on the reference's own 3D fixtures, the march taken by default (the
    fixtures' grids are small)."""
    from cuwave_b200 import Source, simulate

    os.environ["CWB_MARCH3D"] = "1"
    try:
        fx = cases.load(name)
        sim, design = cases.product_sim(fx)
        if sim.N < 16:
            pytest.skip("marches shorter than 16 steps are stepped one launch at a time")
        src = Source(fx["source"], fx["signal"].astype(cases.dtype_of(fx)))
        field, traces = simulate(sim, src, design.copy(), fx["sensors"])
        np.testing.assert_array_equal(traces.cpu().numpy(), fx["traces"])
        np.testing.assert_array_equal(field.cpu().numpy(), fx["field"])
    finally:
        os.environ["CWB_MARCH3D"] = "0"
