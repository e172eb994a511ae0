"""The CPU oracle against the reference's own outputs (tests/golden, make_golden.py).

The oracle restates the reference's kernels in C and its drivers in numpy; run here
it reproduces the reference's CPU fallback bit for bit, forward and adjoint.
"""

import numpy as np
import pytest

import cases
from oracle import oracle as o


@pytest.mark.parametrize("name", cases.FORWARD)
def test_forward_matches_reference(name):
    fx = cases.load(name)
    case = cases.oracle_case(fx)
    field, traces = case.forward(int(fx["N"]))
    Nx = tuple(int(n) for n in fx["Nx"])
    np.testing.assert_array_equal(field[tuple(slice(0, n) for n in Nx)], fx["field"])
    np.testing.assert_array_equal(traces, fx["traces"])


@pytest.mark.parametrize("name", cases.GRADIENT)
def test_gradients_match_reference(name):
    fx = cases.load(name)
    case = cases.oracle_case(fx)
    objective = o.l2(fx["observed"])
    cost, grads, traces = case.sensitivity(int(fx["N"]), objective)
    np.testing.assert_array_equal(traces, fx["traces"])
    np.testing.assert_array_equal(grads["mass"], fx["g_mass"])
    np.testing.assert_array_equal(grads["stiff"], fx["g_stiff"])
    assert cost == pytest.approx(float(fx["cost"]), rel=1e-5)
    _, gradient, _ = case.source_sensitivity(int(fx["N"]), objective)
    np.testing.assert_array_equal(gradient, fx["source_gradient"])


def test_oracle_tables_match_reference():
    tables = np.load(cases.GOLDEN / "stencils.npz")
    for R in range(1, 9):
        for stencil in ("taylor", "optimized"):
            np.testing.assert_allclose(
                o.cell_coefficients(R, stencil), tables[f"coeffs_{stencil}_{R}"], rtol=1e-12, atol=1e-15
            )
            assert o.stable_dt((1.0, 0.5), 1.7, 2 * R, stencil) == pytest.approx(
                float(tables[f"stable_dt_{stencil}_{R}"]), rel=1e-12
            )


def test_planted_error_is_caught():
    """A checker that cannot fail proves nothing: a wrong coefficient must show."""
    fx = cases.load("fwd2d_r4")
    case = cases.oracle_case(fx)
    case.w[1] *= 1.001
    field, _ = case.forward(int(fx["N"]))
    Nx = tuple(int(n) for n in fx["Nx"])
    assert not np.array_equal(field[tuple(slice(0, n) for n in Nx)], fx["field"])


@pytest.mark.parametrize("name", ["fwd2d_r4_pml", "fwd3d_r4_pml"])
def test_float32_error_against_float64(name):
    """The float32 scheme against a float64 run of the same scheme on the same inputs.

    The CUDA path equals the reference's float32 path to the bit (the GPU parity tests),
    so this is the error of both against float64: a few 1e-7 relative L2 here (2D R=4
    with a pml: ~4e-7 of the field; 3D: ~1e-6), far inside the 1e-5 parity bar.
    """
    fx = cases.load(name)
    c32 = cases.oracle_case(fx)
    f32, t32 = c32.forward(int(fx["N"]))
    c64 = cases.oracle_case(fx, dtype=np.float64)
    f64, t64 = c64.forward(int(fx["N"]))
    err = np.linalg.norm(f32.astype(np.float64) - f64) / np.linalg.norm(f64)
    terr = np.linalg.norm(t32.astype(np.float64) - t64) / np.linalg.norm(t64)
    assert 0 < err < 1e-5 and 0 < terr < 1e-5, (err, terr)


REF_CASES = ["fwd2d_r4", "fwd2d_r4_f64", "fwd2d_r4_pml", "fwd3d_r4_pml"]


@pytest.mark.parametrize("level", ["v1", "v3", "v4"])
@pytest.mark.parametrize("name", REF_CASES)
def test_reference_build_matches_reference(name, level):
    """oracle/_ref (the reference's own kernels, compiled by oracle/ref_build.py at each
    instruction-set level) against the fixtures the reference's Python produced: bit for
    bit, forward field and traces, so the CPU baseline and the large-grid parity checks
    that use it run the reference's arithmetic."""
    import importlib.util
    import os

    spec = importlib.util.spec_from_file_location("_rb", cases.ROOT / "oracle" / "ref_build.py")
    rb = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rb)
    fx = cases.load(name)
    tag = "f32" if str(fx["precision"]) == "float32" else "f64"
    ndim = int(fx["ndim"])
    path = rb.library_name(ndim, 4, "optimized", str(fx["precision"]), level)
    if not path.exists():
        pytest.skip(f"{path.name} not built (oracle/ref_build.py needs the reference tree)")
    need = dict((t, f) for t, _, f in rb.LEVELS)[level]
    if not all(f in rb.host_flags() for f in need):
        pytest.skip(f"this host cannot run {level} code")
    case = cases.oracle_case(fx)
    lib = o.ctypes.CDLL(str(path))
    assert lib.ref_ndim() == ndim and tag in path.name
    field, traces = o.ref_simulate(case, int(fx["N"]), threads=min(4, os.cpu_count() or 1),
                                   library=path)
    Nx = tuple(int(n) for n in fx["Nx"])
    np.testing.assert_array_equal(field[tuple(slice(0, n) for n in Nx)], fx["field"])
    np.testing.assert_array_equal(traces, fx["traces"])


SUPERPOSITION = sorted(p.stem for p in cases.GOLDEN.glob("sup*.npz"))


@pytest.mark.parametrize("name", SUPERPOSITION)
def test_superposition_matches_reference(name):
    """The three-slot superposition adjoint, bit for bit with the reference's."""
    fx = cases.load(name)
    case = cases.oracle_case(fx)
    scale = float(fx["scale"])
    cost, grads, traces, cancellation = case.superposition(
        int(fx["N"]), o.l2(fx["observed"]), scale=scale)
    np.testing.assert_array_equal(traces, fx["traces"])
    np.testing.assert_array_equal(grads["mass"], fx["g_mass"])
    np.testing.assert_array_equal(grads["stiff"], fx["g_stiff"])
    assert cost == pytest.approx(float(fx["cost"]), rel=1e-5)
    assert cancellation == pytest.approx(float(fx["cancellation"]), rel=1e-3)


def test_superposition_cancellation_tracks_the_scale():
    """The cancellation B(w, w) - B(u, u) leaves scales as 1 / k while the cross term
    dominates the k^2 one (cuwave sensitivity_test.py:847-855)."""
    fx = cases.load("sup2d_r4_f64")
    objective = o.l2(fx["observed"])
    N = int(fx["N"])
    loose = cases.oracle_case(fx).superposition(N, objective, scale=10.0)[3]
    tight = cases.oracle_case(fx).superposition(N, objective, scale=100.0)[3]
    assert loose / tight == pytest.approx(10.0, rel=0.03)


SPECTRAL = sorted(p.stem for p in cases.GOLDEN.glob("spec*.npz"))


def _spectral_case(fx):
    case = cases.oracle_case(fx)
    region = fx["region"] if fx["region"].size else None
    coef = fx["coef"]

    def linear(traces):
        return float(np.sum(coef * traces)), coef.copy()

    return case, region, linear


@pytest.mark.parametrize("name", SPECTRAL)
def test_spectral_matches_reference(name):
    """The spectral adjoint (running DFTs, decaying adjoint pulses), bit for bit with the
    reference's under a cost linear in the record."""
    fx = cases.load(name)
    case, region, linear = _spectral_case(fx)
    cost, grads, traces, info = case.spectral(int(fx["N"]), linear, fx["frequencies"], region)
    np.testing.assert_array_equal(traces, fx["traces"])
    np.testing.assert_array_equal(grads["mass"], fx["g_mass"])
    np.testing.assert_array_equal(grads["stiff"], fx["g_stiff"])
    assert cost == pytest.approx(float(fx["cost"]), rel=1e-5)
    assert info["decay"] == pytest.approx(float(fx["decay"]), rel=1e-6)
    assert info["fit"] == pytest.approx(float(fx["fit"]), rel=1e-3, abs=1e-12)


MASKED = sorted(p.stem for p in cases.GOLDEN.glob("mask*.npz"))


def masked_oracle_case(fx):
    """The oracle Case of a masked fixture: its cell codes and table rows."""
    case = cases.oracle_case(fx)
    Nx = tuple(int(n) for n in fx["Nx"])
    stepped = np.ones(o.padded(Nx), bool)
    if fx["domain"].size:
        stepped &= fx["domain"]
    held = fx["dirichlet_mask"] if fx["dirichlet_mask"].size else None
    if held is not None:
        stepped &= ~held
    case.cells = o.domain_cells(Nx, case.R, stepped, held)
    case.table = o.cell_table(case.R, str(fx["stencil"]), case.dtype)
    return case


@pytest.mark.parametrize("name", MASKED)
def test_masked_domain_matches_reference(name):
    """A domain mask graded at its walls and held obstacles, bit for bit: the cell codes,
    the forward run and the signal gradient stepped back by the graded step itself."""
    fx = cases.load(name)
    case = masked_oracle_case(fx)
    Nx = tuple(int(n) for n in fx["Nx"])
    interior = tuple(slice(1, n - 1) for n in Nx)
    np.testing.assert_array_equal(case.cells[interior], fx["cells"][interior])
    field, traces = case.forward(int(fx["N"]))
    np.testing.assert_array_equal(field[tuple(slice(0, n) for n in Nx)], fx["field"])
    np.testing.assert_array_equal(traces, fx["traces"])
    cost, gradient, _ = case.source_sensitivity(int(fx["N"]), o.l2(fx["observed"]))
    np.testing.assert_array_equal(gradient, fx["source_gradient"])
    assert cost == pytest.approx(float(fx["source_cost"]), rel=1e-5)
