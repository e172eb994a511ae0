"""Generate the golden fixtures by running the reference package itself.

Runs cmpmech/cuwave from its source tree on its CPU fallback (the same scalar.cu /
scalar_sensitivity.cu kernels, compiled for the host by g++ with OpenMP) on small
seeded cases, and stores the inputs with the outputs in tests/golden/*.npz. The tests
rebuild each case from the stored inputs and compare the oracle (and, on a GPU, the
CUDA path) against the stored outputs.

    python tests/golden/make_golden.py [--reference PATH]

Needs the reference source tree; nothing at test time reads it.
"""

from __future__ import annotations

import argparse
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def setup(reference: str) -> None:
    os.environ["CUWAVE_DEVICE"] = "cpu"
    # the image default CXX lacks libgomp; the system g++ has it
    os.environ["CXX"] = os.environ.get("GOLDEN_CXX", "/usr/bin/g++")
    os.environ.setdefault("XDG_CACHE_HOME", tempfile.mkdtemp(prefix="cuwave-golden-"))
    os.environ.setdefault("OMP_NUM_THREADS", "8")
    sys.path.insert(0, reference)


def smooth_indicator(rng, shape, blobs=4):
    """A smooth field in [0, 1]: a few Gaussian bumps."""
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    out = np.zeros(shape)
    for _ in range(blobs):
        centre = [rng.uniform(0, n) for n in shape]
        sigma = rng.uniform(2.0, max(3.0, min(shape) / 4))
        r2 = sum((g - c) ** 2 for g, c in zip(grids, centre))
        out += rng.uniform(0.3, 1.0) * np.exp(-r2 / (2 * sigma**2))
    return np.clip(out / max(out.max(), 1e-12), 0.0, 1.0)


def stencil_tables():
    from cuwave.stencils import cell_coefficients
    from cuwave.wave import stable_dt

    out = {}
    for R in range(1, 9):
        for stencil in ("taylor", "optimized"):
            out[f"coeffs_{stencil}_{R}"] = cell_coefficients(R, stencil)
            out[f"stable_dt_{stencil}_{R}"] = np.array(
                stable_dt((1.0, 0.5), 1.7, 2 * R, stencil)
            )
    return out


def build_case(name, ndim, Nx, order, N, *, faces="neumann", pml=None, damping=False,
               stencil="optimized", scalar=False, precision="float32", nsens=3, seed=0):
    """Inputs of one run: a dict of arrays and scalars, rebuildable without the reference."""
    from cuwave.wave import padded_shape
    from cuwave.signals import ricker
    from cuwave.stencils import cell_coefficients

    rng = np.random.default_rng(seed)
    shape = padded_shape(Nx)
    indicator = np.zeros(shape)
    indicator[tuple(slice(0, n) for n in Nx)] = smooth_indicator(rng, Nx)
    c = cell_coefficients(order // 2, stencil)
    lam = 4.0 * abs(float(c @ (-1.0) ** np.arange(len(c))))
    cmax = 1.0 if scalar else 1.3
    dx = tuple(1.0 for _ in Nx)
    dt = 0.5 * 2.0 / (cmax * np.sqrt(lam * sum(1.0 / d**2 for d in dx)))
    t = np.arange(N) * dt
    freq = 1.0 / (20.0 * dx[0])
    src = np.array([[n // 2] for n in Nx], dtype=np.int32)
    sens = np.stack(
        [rng.integers(2, n - 2, size=nsens) for n in Nx]
    ).astype(np.int32)
    signal = ricker(t, 1.0, freq)[:, None].astype(precision)
    case = dict(
        name=name, ndim=ndim, Nx=np.array(Nx), order=order, N=N, dt=dt, stencil=stencil,
        faces=faces, scalar=scalar, precision=precision, indicator=indicator,
        source=src, signal=signal, sensors=sens, kappa2=1.0 / 1.69,
        pml=np.array(pml if pml is not None else [0, 0.0]), damping=damping,
    )
    return case


def make_sim(case):
    from cuwave.boundary import Dirichlet, Neumann, Pml, sponge
    from cuwave.scalar import AcousticWave, ScalarWave

    Nx = tuple(int(n) for n in case["Nx"])
    ndim = len(Nx)
    if case["faces"] == "neumann":
        boundary = Neumann
    elif case["faces"] == "dirichlet":
        boundary = Dirichlet
    else:  # mixed: Dirichlet on the low face of axis 0 and the high face of the last axis
        boundary = [[Neumann, Neumann] for _ in range(ndim)]
        boundary[0][0] = Dirichlet
        boundary[-1][1] = Dirichlet
        boundary = tuple(tuple(p) for p in boundary)
    pml = None
    if case["pml"][0] > 0:
        pml = Pml(width=int(case["pml"][0]), wavespeed=float(case["pml"][1]))
    common = dict(
        Nx=Nx, dx=tuple(1.0 for _ in Nx), N=int(case["N"]), dt=float(case["dt"]),
        threads=(8,) * (ndim - 1) + (32,), precision=str(case["precision"]),
        space_order=int(case["order"]), stencil=str(case["stencil"]), boundary=boundary,
        pml=pml,
    )
    if case["scalar"]:
        sim = ScalarWave(**common, wavespeed=1.0, density=1.0)
    else:
        sim = AcousticWave(**common, rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=float(case["kappa2"]))
    if case["damping"]:
        from dataclasses import replace

        ind = case["indicator"].astype(sim.dtype) if not case["scalar"] else 1.0 + case["indicator"].astype(sim.dtype)
        damping = sponge(sim, ind.copy(), width=4, beta=0.3)
        sim = replace(sim, damping=damping)
    return sim


def design(case, sim):
    ind = case["indicator"].astype(sim.dtype)
    return (1.0 + ind) if case["scalar"] else ind


def run_forward(case):
    from cuwave.wave import Source, simulate

    sim = make_sim(case)
    source = Source(case["source"].copy(), case["signal"].astype(sim.dtype))
    field, um = simulate(sim, source, design(case, sim).copy(), case["sensors"].copy())
    out = dict(case)
    out["field"] = np.asarray(field)
    out["traces"] = np.asarray(um)
    if sim.damping is not None:
        out["damping_field"] = np.asarray(sim.damping)
    return out


def run_gradients(case):
    from cuwave.sensitivity import (
        l2_misfit,
        reconstruction_sensitivity,
        sensitivity,
        source_sensitivity,
    )
    from cuwave.wave import Source, simulate

    sim = make_sim(case)
    source = Source(case["source"].copy(), case["signal"].astype(sim.dtype))
    # observed traces from a perturbed design
    perturbed = design(case, sim).copy()
    perturbed *= 0.95
    _, observed = simulate(sim, source, perturbed, case["sensors"].copy())
    observed = np.asarray(observed)
    objective = l2_misfit(observed)
    cost, grads, um, _ = sensitivity(sim, source, design(case, sim).copy(), case["sensors"].copy(), objective)
    scost, sgrad, _, _ = source_sensitivity(sim, source, design(case, sim).copy(), case["sensors"].copy(), objective)
    rcost, rgrads, _, info = reconstruction_sensitivity(
        sim, source, design(case, sim).copy(), case["sensors"].copy(), objective, checkpoints=2
    )
    out = dict(case)
    out.update(
        observed=observed, cost=np.array(cost), g_mass=np.asarray(grads["mass"]),
        g_stiff=np.asarray(grads["stiff"]), traces=np.asarray(um), source_cost=np.array(scost),
        source_gradient=np.asarray(sgrad), rec_cost=np.array(rcost),
        rec_g_mass=np.asarray(rgrads["mass"]), rec_g_stiff=np.asarray(rgrads["stiff"]),
        rec_strip=np.array(info["strip"]), rec_segment=np.array(info["segment"]),
        rec_sweeps=np.array(info["sweeps"]),
    )
    if sim.damping is not None:
        out["damping_field"] = np.asarray(sim.damping)
    return out


def run_superposition(case, scale):
    """superposition_sensitivity of cuwave's sensitivity.py on a lossless case."""
    from cuwave.sensitivity import l2_misfit, superposition_sensitivity
    from cuwave.wave import Source, simulate

    sim = make_sim(case)
    source = Source(case["source"].copy(), case["signal"].astype(sim.dtype))
    perturbed = design(case, sim).copy()
    perturbed *= 0.95
    _, observed = simulate(sim, source, perturbed, case["sensors"].copy())
    observed = np.asarray(observed)
    cost, grads, um, info = superposition_sensitivity(
        sim, source, design(case, sim).copy(), case["sensors"].copy(), l2_misfit(observed),
        scale=scale,
    )
    out = dict(case)
    out.update(
        observed=observed, scale=np.array(scale), cost=np.array(cost), traces=np.asarray(um),
        g_mass=np.asarray(grads["mass"]), g_stiff=np.asarray(grads["stiff"]),
        cancellation=np.array(info["cancellation"]),
    )
    return out


def spectral_coefficients(case, frequencies, dt, seed=11):
    """(N, nsens) sinusoids at `frequencies`: the derivative of a cost linear in the record."""
    rng = np.random.default_rng(seed)
    N, nsens = int(case["N"]), case["sensors"].shape[1]
    t = np.arange(N) * dt
    coef = np.zeros((N, nsens))
    for f in frequencies:
        a, b = rng.standard_normal((2, nsens))
        coef += a * np.cos(2 * np.pi * f * t)[:, None] + b * np.sin(2 * np.pi * f * t)[:, None]
    return coef.astype(case["precision"])


def run_spectral(case, frequencies, box=None):
    """spectral_sensitivity of cuwave's sensitivity.py, under a cost linear in the record
    (its derivative an input, so the whole run is deterministic) and under `intensity`."""
    from cuwave.sensitivity import spectral_sensitivity
    from cuwave.utils import intensity
    from cuwave.wave import Source

    sim = make_sim(case)
    source = Source(case["source"].copy(), case["signal"].astype(sim.dtype))
    coef = spectral_coefficients(case, frequencies, sim.dt)

    def linear(traces):
        return float(np.sum(coef * traces)), coef.copy()

    region = None
    if box is not None:
        region = np.zeros(sim.Nx_padded, dtype=bool)
        region[tuple(slice(lo, hi) for lo, hi in box)] = True
    out = dict(case)
    out.update(frequencies=np.array(frequencies), coef=coef,
               region=region if region is not None else np.zeros(0, bool))
    for tag, objective in (("", linear), ("i_", intensity(sim, frequencies))):
        cost, grads, um, info = spectral_sensitivity(
            sim, source, design(case, sim).copy(), case["sensors"].copy(), objective,
            frequencies, region,
        )
        out.update({
            f"{tag}cost": np.array(cost), f"{tag}traces": np.asarray(um),
            f"{tag}g_mass": np.asarray(grads["mass"]), f"{tag}g_stiff": np.asarray(grads["stiff"]),
            f"{tag}decay": np.array(info["decay"]), f"{tag}fit": np.array(info["fit"]),
        })
    if sim.damping is not None:
        out["damping_field"] = np.asarray(sim.damping)
    return out


def masks(case, kind):
    """(domain, dirichlet) boolean masks over the padded grid: a disk or ball, an obstacle
    held at zero inside it, or a held row across the box."""
    from cuwave.wave import padded_shape

    Nx = tuple(int(n) for n in case["Nx"])
    shape = padded_shape(Nx)
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    centre = [(n - 1) / 2 for n in Nx]
    r2 = sum((g - c) ** 2 for g, c in zip(grids, centre))
    radius = 0.45 * min(Nx)
    domain = dirichlet = None
    if kind in ("disk", "obstacle"):
        domain = r2 <= radius**2
    if kind == "obstacle":
        off = [c + 0.3 * radius * (1 if d == 0 else -1) for d, c in enumerate(centre)]
        dirichlet = sum((g - c) ** 2 for g, c in zip(grids, off)) <= (0.25 * radius) ** 2
    if kind == "row":
        dirichlet = np.zeros(shape, bool)
        dirichlet[int(0.7 * Nx[0])] = True
    return domain, dirichlet


def run_masked(case, kind):
    """simulate and source_sensitivity of cuwave on a masked domain."""
    from cuwave.sensitivity import l2_misfit, source_sensitivity
    from cuwave.wave import Source, domain_cells, simulate

    sim = make_sim(case)
    domain, dirichlet = masks(case, kind)
    sim.domain, sim.dirichlet = domain, dirichlet
    Nx = tuple(int(n) for n in case["Nx"])
    centre = [n // 2 for n in Nx]
    src = np.array([[c] for c in centre], np.int32)
    offsets = [(-3, 2, -4), (1, -1, 2), (-2, 3, 4)]
    offsets = offsets[:1] + offsets[1:-1][: len(Nx) - 2] + offsets[-1:]
    sens = np.array([[c + o for o in offs] for c, offs in zip(centre, offsets)], np.int32)
    source = Source(src, case["signal"].astype(sim.dtype))
    field, um = simulate(sim, source, design(case, sim).copy(), sens.copy())
    observed = np.asarray(um) * sim.dtype(0.7)
    cost, gradient, _, _ = source_sensitivity(
        sim, source, design(case, sim).copy(), sens.copy(), l2_misfit(observed))
    out = dict(case)
    out.update(
        kind=kind, domain=domain if domain is not None else np.zeros(0, bool),
        dirichlet_mask=dirichlet if dirichlet is not None else np.zeros(0, bool),
        source=src, sensors=sens, field=np.asarray(field), traces=np.asarray(um),
        observed=observed, source_cost=np.array(cost), source_gradient=np.asarray(gradient),
        cells=np.asarray(domain_cells(sim)),
    )
    return out


def run_glue(case, shot_coords, receiver_coords):
    """The shot glue of cuwave utils.py on off-node shots and receivers."""
    from cuwave.sensitivity import l2_misfit, reconstruction_sensitivity, source_sensitivity
    from cuwave.utils import (
        Sensors, collect_source, energy, measure, misfit, misfit_gradient, point_source,
        response_gradient, shots, stack,
    )

    sim = make_sim(case)
    signal = case["signal"][:, 0]
    sources = shots(sim, shot_coords, signal)
    sensors = Sensors(sim, receiver_coords)
    perturbed = design(case, sim).copy()
    perturbed *= 0.95
    observed = [np.asarray(o) for o in measure(sim, sources, perturbed, sensors)]
    cost = misfit(sim, sources, design(case, sim).copy(), sensors, observed)
    gcost, gradient = misfit_gradient(sim, sources, design(case, sim).copy(), sensors, observed)
    rcost, rgradient = misfit_gradient(
        sim, sources, design(case, sim).copy(), sensors, observed,
        adjoint=reconstruction_sensitivity,
    )
    stacked = stack(sources)
    stacked_traces = measure(sim, [stacked], design(case, sim).copy(), sensors)[0]
    ecost, egradient = response_gradient(
        sim, stacked, design(case, sim).copy(), sensors.nodes, sensors.objective(energy(sim))
    )
    one = point_source(sim, shot_coords[:1], signal)
    scost, scolumns, _, _ = source_sensitivity(
        sim, one, design(case, sim).copy(), sensors.nodes,
        sensors.objective(l2_misfit(observed[0])),
    )
    out = dict(case)
    out.update(
        shot_coords=np.asarray(shot_coords, dtype=float),
        receiver_coords=np.asarray(receiver_coords, dtype=float),
        sensor_nodes=np.asarray(sensors.nodes), sensor_weights=np.asarray(sensors.weights),
        observed=np.stack(observed), misfit=np.array(cost), gradient_cost=np.array(gcost),
        gradient=np.asarray(gradient), rec_cost=np.array(rcost),
        rec_gradient=np.asarray(rgradient), stacked_position=np.asarray(stacked.position),
        stacked_signal=np.asarray(stacked.signal), stacked_traces=np.asarray(stacked_traces),
        energy_cost=np.array(ecost), energy_gradient=np.asarray(egradient),
        source_cost=np.array(scost), source_columns=np.asarray(scolumns),
        source_signal_gradient=np.asarray(collect_source(sim, shot_coords[:1], scolumns)),
    )
    for k, s in enumerate(sources):
        out[f"shot{k}_position"] = np.asarray(s.position)
        out[f"shot{k}_signal"] = np.asarray(s.signal)
    return out


def run_distribute(name, Nx, dx, precision, seed):
    """`distribute`, `point_source` and `collect_source` alone on a grid of uneven spacing."""
    from cuwave.scalar import AcousticWave
    from cuwave.utils import collect_source, distribute, point_source

    rng = np.random.default_rng(seed)
    ndim = len(Nx)
    sim = AcousticWave(
        Nx=Nx, dx=dx, N=7, dt=0.1, threads=(8,) * (ndim - 1) + (32,), precision=precision,
        space_order=4,
        rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=0.5,
    )
    length = np.array([(n - 3) * d for n, d in zip(Nx, dx)])
    coords = [rng.uniform(0, 1, ndim) * length for _ in range(5)]
    coords += [np.zeros(ndim), length.copy(), length * (1 + 1e-9)]  # walls, just past one
    coords += [np.array([2 * d for d in dx])]  # on a node
    corner = length.copy()
    corner[0] = 0.0
    coords += [corner]
    coords = np.array(coords)
    nodes, weights = distribute(sim, coords)
    scaled_nodes, scaled_weights = distribute(sim, coords, direction=[[-1.5]])
    signal = rng.standard_normal((7, len(coords)))
    source = point_source(sim, coords, signal)
    columns = rng.standard_normal((7, len(coords) * 2**ndim)).astype(sim.dtype)
    collected = collect_source(sim, coords, columns)
    return dict(
        name=name, Nx=np.array(Nx), dx=np.array(dx), precision=precision, coords=coords,
        nodes=np.asarray(nodes), weights=np.asarray(weights),
        scaled_nodes=np.asarray(scaled_nodes), scaled_weights=np.asarray(scaled_weights),
        signal=signal, position=np.asarray(source.position), columns_out=np.asarray(source.signal),
        columns_in=columns, collected=np.asarray(collected),
    )


FORWARD = [
    dict(name="fwd2d_r1", ndim=2, Nx=(30, 37), order=2, N=80),
    dict(name="fwd2d_r2_mixed", ndim=2, Nx=(30, 40), order=4, N=80, faces="mixed"),
    dict(name="fwd2d_r4", ndim=2, Nx=(40, 46), order=8, N=100),
    dict(name="fwd2d_r4_taylor_dir", ndim=2, Nx=(33, 35), order=8, N=70, faces="dirichlet",
         stencil="taylor"),
    dict(name="fwd2d_r8", ndim=2, Nx=(36, 44), order=16, N=60),
    dict(name="fwd2d_r4_damped", ndim=2, Nx=(34, 38), order=8, N=70, damping=True),
    dict(name="fwd2d_r4_pml", ndim=2, Nx=(44, 50), order=8, N=120, pml=(8, 1.3)),
    dict(name="fwd2d_r3_pml_mixed", ndim=2, Nx=(40, 42), order=6, N=90, pml=(6, 1.3),
         faces="mixed"),
    dict(name="fwd2d_scalar_r2", ndim=2, Nx=(30, 33), order=4, N=60, scalar=True),
    dict(name="fwd3d_r1", ndim=3, Nx=(16, 18, 20), order=2, N=40),
    dict(name="fwd3d_r4_pml", ndim=3, Nx=(26, 24, 28), order=8, N=50, pml=(5, 1.3)),
    dict(name="fwd3d_r2_mixed", ndim=3, Nx=(18, 17, 21), order=4, N=40, faces="mixed"),
    dict(name="fwd2d_r4_f64", ndim=2, Nx=(34, 38), order=8, N=70, precision="float64"),
]

GRADIENTS = [
    dict(name="grad2d_r4", ndim=2, Nx=(34, 38), order=8, N=70),
    dict(name="grad2d_r4_pml", ndim=2, Nx=(44, 46), order=8, N=90, pml=(8, 1.3)),
    dict(name="grad2d_r2_mixed", ndim=2, Nx=(30, 33), order=4, N=60, faces="mixed"),
    dict(name="grad2d_r4_damped", ndim=2, Nx=(34, 36), order=8, N=60, damping=True),
    dict(name="grad3d_r2_pml", ndim=3, Nx=(22, 20, 24), order=4, N=40, pml=(5, 1.3)),
    dict(name="grad2d_r4_pml_f64", ndim=2, Nx=(40, 42), order=8, N=70, pml=(7, 1.3),
         precision="float64"),
]


SUPERPOSITION = [
    (dict(name="sup2d_r4", ndim=2, Nx=(34, 38), order=8, N=70), 3e4),
    (dict(name="sup2d_r2_mixed", ndim=2, Nx=(30, 33), order=4, N=60, faces="mixed"), 0.01),
    (dict(name="sup2d_r1_dir_taylor", ndim=2, Nx=(28, 30), order=2, N=50, faces="dirichlet",
          stencil="taylor"), 3e4),
    (dict(name="sup3d_scalar_r2", ndim=3, Nx=(18, 20, 22), order=4, N=40, scalar=True), 1e4),
    (dict(name="sup2d_r4_f64", ndim=2, Nx=(32, 36), order=8, N=60, precision="float64"), 1e3),
]

SPECTRAL = [
    (dict(name="spec2d_r4_pml", ndim=2, Nx=(44, 50), order=8, N=700, pml=(8, 1.3)),
     (0.12, 0.15), None),
    (dict(name="spec2d_r2_damped_region", ndim=2, Nx=(34, 38), order=4, N=700, damping=True),
     (0.12,), ((8, 20), (10, 24))),
    (dict(name="spec3d_r2_pml", ndim=3, Nx=(22, 20, 24), order=4, N=500, pml=(5, 1.3)),
     (0.15,), None),
]

MASKED = [
    (dict(name="mask2d_disk_r2", ndim=2, Nx=(40, 44), order=4, N=120), "disk"),
    (dict(name="mask2d_obstacle_r4_mixed", ndim=2, Nx=(42, 40), order=8, N=110, faces="mixed"),
     "obstacle"),
    (dict(name="mask2d_row_r1_f64", ndim=2, Nx=(36, 34), order=2, N=100, precision="float64"),
     "row"),
    (dict(name="mask2d_obstacle_r6_scalar", ndim=2, Nx=(44, 46), order=12, N=90, scalar=True,
          stencil="taylor"), "obstacle"),
    (dict(name="mask3d_obstacle_r2", ndim=3, Nx=(22, 24, 26), order=4, N=50), "obstacle"),
]

GLUE = [
    (dict(name="glue2d_r4", ndim=2, Nx=(40, 44), order=8, N=80),
     [(12.3, 20.7), (25.6, 9.2)], [(3.5, 2.25 + 7.3 * k) for k in range(6)]),
    (dict(name="glue3d_scalar_r2_pml", ndim=3, Nx=(22, 20, 24), order=4, N=40, pml=(4, 1.0),
          scalar=True),
     [(9.4, 8.1, 10.6)], [(5.5, 5.2, 5.0 + 3.1 * k) for k in range(4)]),
]

DISTRIBUTE = [
    dict(name="distribute2d", Nx=(30, 25), dx=(0.7, 1.3), precision="float32", seed=3),
    dict(name="distribute3d", Nx=(12, 14, 16), dx=(0.5, 0.9, 1.1), precision="float32", seed=4),
    dict(name="distribute2d_f64", Nx=(21, 26), dx=(1.7, 0.3), precision="float64", seed=5),
]


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--reference", default="/root/reference")
    parser.add_argument("--only", default=None)
    args = parser.parse_args(argv)
    setup(args.reference)
    np.savez_compressed(HERE / "stencils.npz", **stencil_tables())
    for spec in FORWARD:
        if args.only and args.only not in spec["name"]:
            continue
        out = run_forward(build_case(**spec))
        np.savez_compressed(HERE / f"{spec['name']}.npz", **out)
        print(spec["name"], "ok", flush=True)
    for spec in GRADIENTS:
        if args.only and args.only not in spec["name"]:
            continue
        out = run_gradients(build_case(**spec))
        np.savez_compressed(HERE / f"{spec['name']}.npz", **out)
        print(spec["name"], "ok", flush=True)
    for spec, scale in SUPERPOSITION:
        if args.only and args.only not in spec["name"]:
            continue
        out = run_superposition(build_case(**spec), scale)
        np.savez_compressed(HERE / f"{spec['name']}.npz", **out)
        print(spec["name"], "ok", flush=True)
    for spec, frequencies, box in SPECTRAL:
        if args.only and args.only not in spec["name"]:
            continue
        out = run_spectral(build_case(**spec), frequencies, box)
        np.savez_compressed(HERE / f"{spec['name']}.npz", **out)
        print(spec["name"], "ok", flush=True)
    for spec, kind in MASKED:
        if args.only and args.only not in spec["name"]:
            continue
        out = run_masked(build_case(**spec), kind)
        np.savez_compressed(HERE / f"{spec['name']}.npz", **out)
        print(spec["name"], "ok", flush=True)
    for spec, shot_coords, receiver_coords in GLUE:
        if args.only and args.only not in spec["name"]:
            continue
        out = run_glue(build_case(**spec), shot_coords, receiver_coords)
        np.savez_compressed(HERE / f"{spec['name']}.npz", **out)
        print(spec["name"], "ok", flush=True)
    for spec in DISTRIBUTE:
        if args.only and args.only not in spec["name"]:
            continue
        out = run_distribute(**spec)
        np.savez_compressed(HERE / f"{spec['name']}.npz", **out)
        print(spec["name"], "ok", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
