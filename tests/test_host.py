"""Host-side logic that needs no GPU: the C ABI surface, setup tables, validation."""

import ctypes
import re
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import cases
from oracle import oracle as o

ROOT = cases.ROOT
HEADER = ROOT / "include" / "cuwave_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:[\w*]+\s+)+\**(cwb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    from cuwave_b200 import _native

    lib = ctypes.CDLL(str(_native.LIBRARY))
    names = declared_functions()
    assert len(names) >= 6
    for name in names:
        assert hasattr(lib, name), name
    assert lib.cwb_version() == 1


def test_ctypes_layout_matches_header():
    """Every struct the binding mirrors has the header's size and field offsets."""
    from cuwave_b200 import _native as nat

    structs = {"cwb_grid": nat.Grid, "cwb_level": nat.Level, "cwb_material": nat.Material,
               "cwb_points": nat.Points, "cwb_op": nat.Op, "cwb_batch_item": nat.BatchItem}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as tmp:
        src = Path(tmp) / "layout.c"
        exe = Path(tmp) / "layout"
        src.write_text("\n".join(lines))
        subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert int(got[f"{cname}.{field}"]) == getattr(py, field).offset, (cname, field)


def test_stencil_tables_match_reference():
    from cuwave_b200 import stencils

    tables = np.load(cases.GOLDEN / "stencils.npz")
    for R in range(1, 9):
        for stencil in ("taylor", "optimized"):
            ref = tables[f"coeffs_{stencil}_{R}"]
            got = stencils.cell_coefficients(R, stencil)
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)
            # the kernels read the float32 rounding: identical bits
            np.testing.assert_array_equal(got.astype(np.float32), ref.astype(np.float32))
            assert stencils.stable_dt((1.0, 0.5), 1.7, 2 * R, stencil) == pytest.approx(
                float(tables[f"stable_dt_{stencil}_{R}"]), rel=1e-12
            )


@pytest.mark.parametrize("name", ["fwd2d_r4_pml", "fwd3d_r4_pml", "grad2d_r4_pml_f64"])
def test_pml_profiles_match_oracle(name):
    from cuwave_b200.boundary import pml_profiles

    fx = cases.load(name)
    sim, _ = cases.product_sim(fx)
    ref = cases.oracle_case(fx).profiles
    for got, want in zip(pml_profiles(sim), ref):
        assert (got is None) == (want is None)
        if got is not None:
            np.testing.assert_array_equal(got, want)


def test_simulation_validation():
    from cuwave_b200 import AcousticWave, Pml

    base = dict(Nx=(20, 20), dx=(1.0, 1.0), N=10, dt=0.1, rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=2.0)
    with pytest.raises(ValueError):
        AcousticWave(**base, space_order=3)
    with pytest.raises(ValueError):
        AcousticWave(**base, stencil="nope")
    with pytest.raises(ValueError):
        AcousticWave(**base, domain=np.ones((20, 20), bool))  # not over the padded grid
    with pytest.raises(ValueError):
        AcousticWave(**base, domain=np.ones((20, 32), bool), pml=Pml(width=4, wavespeed=1.0))
    with pytest.raises(ValueError):
        AcousticWave(**{**base, "Nx": (30, 30)}, domain=np.ones((30, 32), bool), space_order=14)
    assert AcousticWave(**base, domain=np.ones((20, 32), bool)).masked
    with pytest.raises(NotImplementedError):
        AcousticWave(**base, devices=(0, 1))
    with pytest.raises(ValueError):
        AcousticWave(**{**base, "Nx": (6, 20)}, space_order=8)
    with pytest.raises(ValueError):
        AcousticWave(**base, pml=Pml(width=9, wavespeed=1.0), space_order=2)
    with pytest.raises(ValueError):
        AcousticWave(**{**base, "rho1": None})
    sim = AcousticWave(**base, space_order=4)
    assert sim.Nx_padded == (20, 32)
    assert sim.strides == (32, 1)


def test_bfloat16_narrowing_rounds_to_nearest_even():
    import torch

    from cuwave_b200.wave import narrow, widen

    x = torch.tensor([1.0, 1.00390625, 1.01171875, -3.14159, 1e-30, 65504.0], dtype=torch.float32)
    bits = narrow(x, torch.uint16)
    # the same rounding as torch's own bfloat16 cast on finite values
    np.testing.assert_array_equal(
        widen(bits, torch.float32).numpy(), x.to(torch.bfloat16).to(torch.float32).numpy()
    )


def test_checkpoint_schedule_reverses_every_segment():
    from cuwave_b200.sensitivity import checkpoint_schedule

    for segments in range(1, 20):
        for slots in range(0, 4):
            leaves = [a[1] for a in checkpoint_schedule(segments, slots) if a[0] == "leaf"]
            assert leaves == list(range(segments - 1, -1, -1))
