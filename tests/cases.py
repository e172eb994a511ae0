"""Rebuild the golden cases for the oracle and for the CUDA path.

A fixture (tests/golden/*.npz, written by make_golden.py from the reference itself)
stores a case's inputs next to the reference's outputs. `oracle_case` rebuilds it for
the CPU oracle; `product_case` for cuwave_b200.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

FORWARD = sorted(p.stem for p in GOLDEN.glob("fwd*.npz"))
GRADIENT = sorted(p.stem for p in GOLDEN.glob("grad*.npz"))


def load(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def dtype_of(fx) -> type:
    return np.float32 if str(fx["precision"]) == "float32" else np.float64


def face_masks(fx) -> tuple[int, int]:
    """(dirichlet, neumann) bitmasks of the fixture's faces."""
    ndim = int(fx["ndim"])
    every = (1 << (2 * ndim)) - 1
    faces = str(fx["faces"])
    if faces == "neumann":
        dirichlet = 0
    elif faces == "dirichlet":
        dirichlet = every
    else:
        dirichlet = (1 << 0) | (1 << (2 * (ndim - 1) + 1))
    return dirichlet, every & ~dirichlet


def design(fx) -> np.ndarray:
    dt = dtype_of(fx)
    ind = fx["indicator"].astype(dt)
    return (dt(1.0) + ind).astype(dt) if bool(fx["scalar"]) else ind


def flat(fx, position) -> np.ndarray:
    Nx = tuple(int(n) for n in fx["Nx"])
    shape = (*Nx[:-1], (Nx[-1] + 31) // 32 * 32)
    strides = [1] * len(Nx)
    for d in range(len(Nx) - 2, -1, -1):
        strides[d] = strides[d + 1] * shape[d + 1]
    lin = np.zeros(position.shape[1], np.int64)
    for d in range(len(Nx)):
        lin += position[d].astype(np.int64) * strides[d]
    return lin.astype(np.int32)


def oracle_case(fx, dtype=None):
    """The oracle Case of a fixture, in its own precision or in `dtype`."""
    from oracle import oracle as o

    dt_ = dtype_of(fx) if dtype is None else dtype
    Nx = tuple(int(n) for n in fx["Nx"])
    ndim = len(Nx)
    order, dt = int(fx["order"]), float(fx["dt"])
    dirichlet, neumann = face_masks(fx)
    scalar = bool(fx["scalar"])
    if scalar:
        stiff = o.mirror_ghosts(Nx, design(fx).copy())
        minv = None
        factors = [dt_(2.0 * 1.0**2 * dt**2 / 1.0**2)] * ndim
    else:
        stiff, minv = o.acoustic_materials(Nx, design(fx), 1.0, 1.0, 1.0, float(fx["kappa2"]), dt_)
        factors = [dt_(2.0 * dt**2 / 1.0**2)] * ndim
    widths = profiles = None
    if float(fx["pml"][0]) > 0:
        width, speed = int(fx["pml"][0]), float(fx["pml"][1])
        widths = tuple((width, width) for _ in range(ndim))
        profiles = o.pml_profiles(Nx, (1.0,) * ndim, dt, widths, width, speed, 1e-6, 0.0, dt_)
    damping = fx["damping_field"].astype(dt_) if "damping_field" in fx else None
    case = o.Case(
        Nx=Nx, R=order // 2, coeffs=o.cell_coefficients(order // 2, str(fx["stencil"])),
        factors=factors, dt=dt, stiff=stiff, minv=minv, dtype=dt_, dirichlet=dirichlet,
        neumann=neumann, damping=damping, widths=widths, profiles=profiles,
        source_lin=flat(fx, fx["source"]), signal=np.ascontiguousarray(fx["signal"].astype(dt_)),
        sensor_lin=flat(fx, fx["sensors"]),
    )
    case.source_weight = case.excitation_weights(case.source_lin)
    return case


def product_sim(fx):
    """(sim, indicator) of cuwave_b200 for a fixture."""
    from dataclasses import replace

    from cuwave_b200 import AcousticWave, Dirichlet, Neumann, Pml, ScalarWave

    Nx = tuple(int(n) for n in fx["Nx"])
    ndim = len(Nx)
    faces = str(fx["faces"])
    if faces == "neumann":
        boundary = Neumann
    elif faces == "dirichlet":
        boundary = Dirichlet
    else:
        pairs = [[Neumann, Neumann] for _ in range(ndim)]
        pairs[0][0] = Dirichlet
        pairs[-1][1] = Dirichlet
        boundary = tuple(tuple(p) for p in pairs)
    pml = None
    if float(fx["pml"][0]) > 0:
        pml = Pml(width=int(fx["pml"][0]), wavespeed=float(fx["pml"][1]))
    common = dict(
        Nx=Nx, dx=(1.0,) * ndim, N=int(fx["N"]), dt=float(fx["dt"]),
        precision=str(fx["precision"]), space_order=int(fx["order"]),
        stencil=str(fx["stencil"]), boundary=boundary, pml=pml,
    )
    if bool(fx["scalar"]):
        sim = ScalarWave(**common, wavespeed=1.0, density=1.0)
    else:
        sim = AcousticWave(**common, rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=float(fx["kappa2"]))
    if "damping_field" in fx:
        sim = replace(sim, damping=fx["damping_field"].astype(dtype_of(fx)))
    return sim, design(fx)


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / scale) if scale > 0 else float(np.linalg.norm(a - b))
