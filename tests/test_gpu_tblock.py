"""The temporally blocked 2D march (TB_K steps per pass over HBM) against the march that
steps one launch at a time, and against the oracle.

The blocked march recomputes the overlap of neighbouring tiles and row chunks with the
same arithmetic as the single step, so the bar is equality: fields and traces bit for
bit, over grids of several tiles and chunks, every radius it is built for, Neumann,
Dirichlet and mixed faces, sources near walls and tile seams, several receiver sets, and
step counts that are not a multiple of a pass (the rest goes one step at a time).
CWB_TBLOCK=2 takes the blocked path on grids of any size (by default only grids too large
for L2 take it), CWB_TBLOCK=0 turns it off.
"""

import os

import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu


def _sim(Nx, R, N, faces, seed):
    from cuwave_b200 import AcousticWave, Dirichlet, Neumann, stable_dt

    rng = np.random.default_rng(seed)
    if faces == "neumann":
        boundary = Neumann
    elif faces == "dirichlet":
        boundary = Dirichlet
    else:
        boundary = ((Dirichlet, Neumann), (Neumann, Dirichlet))
    c_max = 1.4
    dt = 0.5 * stable_dt((1.0, 1.0), c_max, 2 * R)
    sim = AcousticWave(Nx=Nx, dx=(1.0, 1.0), N=N, dt=dt, precision="float32", space_order=2 * R,
                       boundary=boundary, rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=2.0)
    c = 1.0 + 0.4 * rng.random(Nx)
    ind = np.zeros(sim.Nx_padded, np.float32)
    ind[:, : Nx[1]] = ((1.0 / c**2 - 1.0) / (1.0 / 2.0 - 1.0)).astype(np.float32)
    from cuwave_b200.signals import ricker

    t = np.arange(N) * dt
    # sources near a corner, on a tile seam (x 480 .. 483 at radius <= 4) and inside
    src = np.array([[2, Nx[0] // 2, Nx[0] - 4], [3, min(481, Nx[1] - 3), Nx[1] // 3]], np.int32)
    sig = np.stack([ricker(t, 1.0, 0.08), -0.5 * ricker(t, 1.0, 0.05), ricker(t - 3, 0.3, 0.1)], 1)
    rows = np.full(40, Nx[0] // 3)
    sens = np.stack([rows, np.linspace(1, Nx[1] - 2, 40).round()]).astype(np.int32)
    return sim, ind, src, sig.astype(np.float32), sens


def _run(sim, ind, src, sig, sens, mode):
    """simulate with the blocked path forced (2) or off (0); returns field, traces and the
    launches the march made."""
    from dataclasses import replace

    from cuwave_b200 import Source, _native as nat, simulate

    os.environ["CWB_TBLOCK"] = str(mode)
    try:
        fresh = replace(sim)  # a new plan, made under this setting
        n0 = nat.launches()
        field, traces = simulate(fresh, Source(src, sig), ind.copy(), sens)
        torch.cuda.synchronize()
        return field.cpu().numpy(), traces.cpu().numpy(), nat.launches() - n0
    finally:
        os.environ.pop("CWB_TBLOCK", None)


@pytest.mark.parametrize("R,faces,Nx,N", [
    (4, "neumann", (300, 520), 37),
    (4, "mixed", (170, 1000), 30),
    (3, "dirichlet", (140, 530), 22),
    (2, "mixed", (200, 490), 41),
    (1, "neumann", (90, 600), 13),
])
def test_blocked_march_matches_single_steps(R, faces, Nx, N):
    sim, ind, src, sig, sens = _sim(Nx, R, N, faces, seed=R)
    f_ref, t_ref, l_ref = _run(sim, ind, src, sig, sens, 0)
    f_blk, t_blk, l_blk = _run(sim, ind, src, sig, sens, 2)
    # the blocked path launches one kernel a pass (the rest of the steps one at a time)
    assert l_blk != l_ref and l_blk >= N // 4, (l_blk, l_ref)
    assert np.abs(f_ref).max() > 0
    np.testing.assert_array_equal(t_blk, t_ref)
    np.testing.assert_array_equal(f_blk, f_ref)


def test_blocked_march_matches_oracle():
    """Against the CPU oracle's restatement of the reference's step sequence."""
    sim, ind, src, sig, sens = _sim((130, 530), 4, 25, "neumann", seed=7)
    f_blk, t_blk, _ = _run(sim, ind, src, sig, sens, 2)
    from oracle import oracle as o

    Nx = sim.Nx
    stiff, minv = o.acoustic_materials(Nx, ind, 1.0, 1.0, 1.0, 2.0, np.float32)
    shape = sim.Nx_padded
    flat = lambda p: (p[0].astype(np.int64) * shape[1] + p[1]).astype(np.int32)  # noqa: E731
    case = o.Case(Nx=Nx, R=4, coeffs=o.cell_coefficients(4, "optimized"),
                  factors=[np.float32(2.0 * sim.dt**2)] * 2, dt=sim.dt, stiff=stiff, minv=minv,
                  dtype=np.float32, source_lin=flat(src), signal=sig, sensor_lin=flat(sens))
    case.source_weight = case.excitation_weights(case.source_lin)
    field, traces = case.forward(sim.N)
    np.testing.assert_array_equal(t_blk, traces)
    np.testing.assert_array_equal(f_blk, field[:, : Nx[1]])


@pytest.mark.parametrize("R,dirichlet,pml", [(4, 0b0000, 20), (3, 0b0110, 7), (2, 0b1001, 12),
                                             (1, 0b0000, 5)])
def test_blocked_march_with_pml_matches_oracle(R, dirichlet, pml):
    """With pml slabs on every face (their memory advanced level by level inside the pass,
    around the ring of copies), Dirichlet and Neumann faces, sources anywhere in the
    interior: the oracle's fields and traces, bit for bit, and the single-step march's."""
    from cuwave_b200 import _native as nat
    from test_gpu_parity import _product, _random_case

    case, meta = _random_case(2, R, dirichlet=dirichlet, pml=pml, uniform=True, seed=50 + R,
                              nsrc=4, nsens=9, Nx=(150, 530))
    counts = {}
    results = {}
    for mode in ("0", "2"):
        os.environ["CWB_TBLOCK"] = mode
        try:
            n0 = nat.launches()
            results[mode] = _product(case, meta)
            torch.cuda.synchronize()
            counts[mode] = nat.launches() - n0
        finally:
            os.environ.pop("CWB_TBLOCK", None)
    assert counts["2"] != counts["0"], counts
    ref_field, ref_traces = case.forward(meta["N"])
    for mode in ("0", "2"):
        field, traces = results[mode]
        np.testing.assert_array_equal(traces, ref_traces)
        np.testing.assert_array_equal(field, ref_field)
