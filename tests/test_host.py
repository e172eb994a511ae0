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


def test_checkpoint_schedule_keeps_its_snapshot_budget():
    """Every snapshot stored is dropped again, no more than `slots` are held at once, a
    march starts from the state just restored, and treeverse's replay count is the
    binomial bound's: a segment is re-marched at most r + 1 times for the fewest r with
    C(slots + r, slots) >= segments."""
    import math

    from cuwave_b200.sensitivity import checkpoint_schedule

    for segments in range(1, 60):
        for slots in range(0, 5):
            held, restored, marched = set(), None, [0] * segments
            for action in checkpoint_schedule(segments, slots):
                if action[0] == "store":
                    held.add(action[1])
                    assert len(held) <= slots
                elif action[0] == "drop":
                    held.remove(action[1])
                elif action[0] == "restore":
                    assert action[1] == 0 or action[1] in held
                    restored = action[1]
                elif action[0] == "advance":
                    assert action[1] == restored
                    for k in range(action[1], action[2]):
                        marched[k] += 1
            assert not held
            if slots:
                r = next(r for r in range(segments + 1) if math.comb(slots + r, slots) >= segments)
                assert max(marched) <= r
            else:
                assert max(marched) == segments - 1


def test_resample_and_threshold():
    import torch

    from cuwave_b200.utils import resample, threshold

    x = np.arange(11, dtype=np.float64) * 0.5 + 1.0  # linear: interpolation is exact
    y = resample(x, 1.0, 0.25)
    np.testing.assert_allclose(y, 1.0 + 0.5 * 0.25 * np.arange(41), rtol=0, atol=1e-12)
    z = resample(torch.as_tensor(x), 1.0, 0.5, N_new=30)
    assert torch.all(z[21:] == 0) and float(z[20]) == x[-1]
    field = np.array([0.1, 0.5, 0.7, np.nan], np.float32)
    np.testing.assert_array_equal(threshold(field), np.array([0, 1, 1, 1], np.float32))
    assert threshold(field).dtype == np.float32
    assert torch.equal(threshold(torch.as_tensor(field), 0.6, 0.3, 1.0),
                       torch.tensor([0.3, 0.3, 1.0, 1.0], dtype=torch.float32))


def test_time_dispersion_round_trip():
    """itdt undoes tdt on a signal whose band leapfrog carries, to the truncation of the
    finite transforms (1e-4 of the peak)."""
    import warnings

    from cuwave_b200 import AcousticWave
    from cuwave_b200.signals import ricker
    from cuwave_b200.utils import itdt, leapfrog_frequency, tdt

    sim = AcousticWave(Nx=(20, 20), dx=(1.0, 1.0), N=400, dt=0.2, space_order=4,
                       rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=2.0)
    s = ricker(np.arange(400) * sim.dt, 1.0, 0.2)[:, None]
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        back = itdt(sim, tdt(sim, s, offset=0), offset=0)
        np.testing.assert_allclose(back, s, rtol=0, atol=2e-4 * np.abs(s).max())
        f = leapfrog_frequency(sim, 0.2)
        assert f > 0.2 and np.isclose(np.sin(np.pi * f * sim.dt), np.pi * 0.2 * sim.dt)
