#!/usr/bin/env python
"""Benchmark of the scalar-wave hot path: the 3D forward with PML.

Workload (one bench step = one whole job): AcousticWave on a 512^3 grid (ghosts
included), fp32, radius-4 optimized stencil, 20-cell PML on every face, 4000 leapfrog
steps at CFL 0.5, six seeded horizontal layers of speed in [1.0, 2.5] with a +-5% random
perturbation, a Ricker source at node (22, 256, 256), and a 128 x 128 receiver plane on
row 30 (stride-4 columns). Data are synthetic (seeded), inputs larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is Gpt-updates/s (interior nodes x time steps / job time) with the inputs
resident in HBM; `e2e` is the same through the public `simulate` call with host
buffers (pinned host -> device copies of the inputs and device -> host copies of the
traces and the final field inside the timed region). Multi-GPU runs are replicas (the
path does not shard across GPUs here): every rank runs the whole job on its own GPU.
`--impl reference` times the reference's own kernels compiled for the host cores
(oracle/_ref) on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gpt-updates/s + % HBM roofline; learned-vs-plain time at 1e-2 rel. trace error"
UNIT = "Gpt-updates/s"
BYTES_PER_UPDATE = 16  # read u^(t-1), u^(t-2), 1/m; write u^t (stiffness uniform)
PML_BYTES = 24  # read + write of psi+, psi-, zeta per slab node per lined axis


def workload(size: int = 512, steps: int = 4000, width: int = 20, seed: int = 0) -> dict:
    """The seeded inputs of the layered 3D job, all numpy."""
    rng = np.random.default_rng(seed)
    Nx = (size, size, size)
    shape = (size, size, (size + 31) // 32 * 32)
    # six layers along axis 0, speeds sorted upwards in depth
    speeds = np.sort(rng.uniform(1.0, 2.5, 6))
    cuts = np.sort(rng.choice(np.arange(2, size - 2), 5, replace=False))
    layer = np.searchsorted(cuts, np.arange(size), side="right")
    c = speeds[layer][:, None, None] * (1.0 + rng.uniform(-0.05, 0.05, Nx))
    c_max = float(c.max())
    kappa2 = 2.5**2
    # AcousticWave with rho1 = rho2 = kappa1 = 1: minv = kappa(gamma) = c^2
    indicator = np.zeros(shape, np.float32)
    indicator[:, :, :size] = ((1.0 / c**2 - 1.0) / (1.0 / kappa2 - 1.0)).astype(np.float32)
    from cuwave_b200.stencils import stable_dt

    dt = 0.5 * stable_dt((1.0, 1.0, 1.0), c_max, 8, "optimized")
    from cuwave_b200.signals import ricker

    freq = float(c.min()) / 20.0
    signal = ricker(np.arange(steps) * dt, 1.0, freq)[:, None].astype(np.float32)
    source = np.array([[22], [size // 2], [size // 2]], np.int32)
    cols = 2 + 4 * np.arange(min(128, (size - 4) // 4))
    a1, a2 = np.meshgrid(cols, cols, indexing="ij")
    sensors = np.stack([np.full(a1.size, 30), a1.ravel(), a2.ravel()]).astype(np.int32)
    return dict(Nx=Nx, steps=steps, width=width, dt=dt, c_max=c_max, kappa2=kappa2,
                indicator=indicator, signal=signal, source=source, sensors=sensors)


def make_sim(w: dict):
    from cuwave_b200 import AcousticWave, Pml

    return AcousticWave(
        Nx=w["Nx"], dx=(1.0, 1.0, 1.0), N=w["steps"], dt=w["dt"], precision="float32",
        space_order=8, stencil="optimized",
        pml=Pml(width=w["width"], wavespeed=w["c_max"]) if w["width"] else None,
        rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=w["kappa2"],
    )


def interior_updates(w: dict) -> int:
    return int(np.prod([n - 2 for n in w["Nx"]]))


def algorithmic_bytes(w: dict) -> int:
    """Compulsory HBM bytes of one time step: 16 B per interior update plus 24 B per pml
    slab node per lined axis."""
    n = [x - 2 for x in w["Nx"]]
    slab = sum(2 * w["width"] * int(np.prod([n[e] for e in range(3) if e != d])) for d in range(3))
    return BYTES_PER_UPDATE * interior_updates(w) + PML_BYTES * slab


# ------------------------------------------------------------------- clocks
REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    def __init__(self, index: int):
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])
        query = "index,clocks.sm,clocks.max.sm,power.draw," + ",".join(
            f"clocks_event_reasons.{r}" for r in REASONS
        )
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), f"--query-gpu={query}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL,
            )
        except FileNotFoundError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(", ") for r in self.path.read_text().splitlines() if r.strip()]
        self.path.unlink(missing_ok=True)
        sm = [float(r[1]) for r in rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) >= 8 and r[2].replace(".", "").isdigit()]
        reasons = sorted({REASONS[i] for r in rows if len(r) >= 8 for i in range(4)
                          if r[4 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------------------- helpers
def dist_setup():
    """(rank, world, local_rank) from the torchrun environment; a gloo/nccl group when > 1."""
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def cpu_baseline(w: dict, sample_steps: int, cores: int | None = None):
    """The reference's own kernels (oracle/_ref, built from its sources) on the host cores,
    a bounded sample of `sample_steps` steps of the same job. Returns the baseline entry
    and the sample's final field and traces (None when the build is missing)."""
    from oracle import oracle as o

    path, level = o.ref_library(3, 4, "optimized", "float32")
    if not path.exists():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": f"unavailable: {path.name} not built (oracle/ref_build.py)"}, None, None
    cores = cores or os.cpu_count() or 1
    case = reference_case(w)
    o.ref_simulate(case, 1, threads=cores)  # page in, spawn the OpenMP team
    t0 = time.perf_counter()
    field, traces = o.ref_simulate(case, sample_steps, threads=cores)
    elapsed = time.perf_counter() - t0
    value = interior_updates(w) * sample_steps / elapsed / 1e9
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{sample_steps} of {w['steps']} steps of the full {w['Nx'][0]}^3 job "
                      f"({elapsed:.1f} s), reference kernels via oracle/_ref built with g++ -O3 "
                      f"-fopenmp -ffp-contract=off -march={REF_MARCH[level]}, OpenMP"}, field, traces


# the -march of each instruction-set level oracle/ref_build.py builds (the reference's own
# host build uses -march=native, cuwave/cpu.py:22)
REF_MARCH = {"v4": "x86-64-v4 (AVX-512)", "v3": "x86-64-v3 (AVX2)", "v1": "x86-64"}


def sample_parity(sim, w: dict, steps: int, ref_field, ref_traces) -> dict:
    """The repo's march over the first `steps` steps of the job (the public `simulate`,
    the same inputs) against the reference kernels' sample: field and traces compared
    to the bit."""
    from dataclasses import replace

    import torch

    from cuwave_b200 import Source, simulate

    dev = torch.device("cuda")
    short = replace(sim, N=steps)
    field, traces = simulate(short, Source(torch.as_tensor(w["source"], device=dev),
                                           torch.as_tensor(w["signal"], device=dev)),
                             torch.as_tensor(w["indicator"], device=dev), torch.as_tensor(w["sensors"], device=dev))
    field = field.cpu().numpy()
    traces = traces.cpu().numpy()
    ref = ref_field[tuple(slice(0, n) for n in w["Nx"])]
    diff = np.abs(field.astype(np.float64) - ref)
    scale = float(np.linalg.norm(ref.astype(np.float64)))
    return {"steps": steps, "field_max_abs": float(diff.max()),
            "field_rel_l2": float(np.linalg.norm(diff) / scale) if scale else float(np.linalg.norm(diff)),
            "traces_max_abs": float(np.abs(traces.astype(np.float64) - ref_traces).max()),
            "bitwise": bool(np.array_equal(field, ref) and np.array_equal(traces, ref_traces)),
            "against": "the cpu_baseline sample (reference kernels via oracle/_ref)"}


def reference_case(w: dict, dtype=np.float32):
    """A 2D or 3D job as an oracle case: the same materials, tables and source weights,
    in `dtype` (the float64 case is the same scheme on the same inputs)."""
    from oracle import oracle as o

    Nx = tuple(w["Nx"])
    ndim = len(Nx)
    R = w.get("radius", 4)
    stiff, minv = o.acoustic_materials(Nx, w["indicator"], 1.0, 1.0, 1.0, w["kappa2"], dtype)
    widths = tuple((w["width"], w["width"]) for _ in range(ndim)) if w["width"] else None
    profiles = o.pml_profiles(Nx, (1.0,) * ndim, w["dt"], widths, w["width"], w["c_max"], 1e-6, 0.0,
                              dtype) if w["width"] else None
    shape = (*Nx[:-1], (Nx[-1] + 31) // 32 * 32)
    strides = [int(np.prod(shape[d + 1:])) for d in range(ndim)]

    def flat(p):
        return sum(p[d].astype(np.int64) * strides[d] for d in range(ndim)).astype(np.int32)

    case = o.Case(Nx=Nx, R=R, coeffs=o.cell_coefficients(R, "optimized"),
                  factors=[dtype(2.0 * w["dt"] ** 2)] * ndim, dt=w["dt"], stiff=stiff, minv=minv,
                  dtype=dtype, widths=widths, profiles=profiles, source_lin=flat(w["source"]),
                  signal=w["signal"].astype(dtype), sensor_lin=flat(w["sensors"]))
    case.source_weight = case.excitation_weights(case.source_lin)
    return case


def blob_workload(n: int, steps: int, width: int = 0, seed: int = 0) -> dict:
    """The 2D blob job: AcousticWave on an n x n grid (ghosts included), radius 4, speed 1
    plus 8 seeded Gaussian blobs (blob_speed), dt at CFL 0.5 of the fastest speed, a Ricker
    source at the centre with about 20 points a wavelength at the slowest speed, 64
    receivers on row 51 at columns linspace(1, n - 2, 64) rounded, an optional pml."""
    from cuwave_b200.signals import ricker
    from cuwave_b200.stencils import stable_dt

    c = blob_speed(n, seed)
    kappa2 = 0.25
    shape = (n, (n + 31) // 32 * 32)
    indicator = np.zeros(shape, np.float32)
    indicator[:, :n] = ((1.0 / c**2 - 1.0) / (1.0 / kappa2 - 1.0)).astype(np.float32)
    c_max = float(c.max())
    dt = 0.5 * stable_dt((1.0, 1.0), c_max, 8, "optimized")
    signal = ricker(np.arange(steps) * dt, 1.0, float(c.min()) / 20.0)[:, None].astype(np.float32)
    source = np.array([[n // 2], [n // 2]], np.int32)
    cols = np.round(np.linspace(1, n - 2, 64)).astype(np.int32)
    sensors = np.stack([np.full(64, 51, np.int32), cols]).astype(np.int32)
    return dict(Nx=(n, n), steps=steps, width=width, dt=dt, c_max=c_max, kappa2=kappa2,
                indicator=indicator, signal=signal, source=source, sensors=sensors, speed=c)


def sensitivity_workload(n: int = 2048, steps: int = 300, width: int = 20, seed: int = 0) -> dict:
    """The 2D gradient job: the blob job on an n x n grid with a `width`-cell pml, one
    source 20 rows inside the pml's inner edge and 256 receivers 40 rows below it
    (columns spread over the interior), and observed traces made with the speed
    perturbed by 5% seeded blobs (c_obs = c (1 + 0.05 b), b a second blob field scaled to
    [-1, 1]), so the misfit is not small. `steps` is short of a full run, so the
    source and the receivers sit close enough for the wave to reach them."""
    w = blob_workload(n, steps, width, seed)
    R = 4
    w["source"] = np.array([[width + 20], [n // 2]], np.int32)
    cols = np.round(np.linspace(width + R + 2, n - width - R - 3, 256)).astype(np.int32)
    w["sensors"] = np.stack([np.full(256, width + 60, np.int32), cols]).astype(np.int32)
    b = (blob_speed(n, seed + 1) - 1.0) / 0.3
    c_obs = w["speed"] * (1.0 + 0.05 * b)
    ind = np.zeros_like(w["indicator"])
    ind[:, :n] = ((1.0 / c_obs**2 - 1.0) / (1.0 / w["kappa2"] - 1.0)).astype(np.float32)
    w["indicator_obs"] = ind
    return w


def make_sim_2d(w: dict, precision: str = "float32", steps: int | None = None):
    from cuwave_b200 import AcousticWave, Pml

    return AcousticWave(
        Nx=w["Nx"], dx=(1.0, 1.0), N=steps or w["steps"], dt=w["dt"], precision=precision,
        space_order=8, stencil="optimized",
        pml=Pml(width=w["width"], wavespeed=w["c_max"]) if w["width"] else None,
        rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=w["kappa2"],
    )


def run_reference(args) -> int:
    rank, world, _ = dist_setup()
    if rank != 0:
        return 0
    w = workload(args.size, args.nt, args.pml)
    sample = args.ref_sample
    times = []
    from oracle import oracle as o

    path, level = o.ref_library(3, 4, "optimized", "float32")
    if not path.exists():
        print(json.dumps({"impl": "reference", "unavailable": f"{path.name} was not built"}))
        return 0
    case = reference_case(w)
    cores = os.cpu_count() or 1
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        o.ref_simulate(case, sample, threads=cores)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    per = sum(times) / len(times)
    value = interior_updates(w) * sample / per / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered model)",
        "config": config_line(w, args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{sample} of {w['steps']} steps of the full job per bench step, "
                                   f"reference kernels via oracle/_ref built with g++ -O3 -fopenmp "
                                   f"-ffp-contract=off -march={REF_MARCH[level]}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def config_line(w: dict, args) -> dict:
    return {"workload": "3D scalar forward with PML (layered 512^3, radius 4, 20-cell PML, "
                        "4000 steps, 128x128 receiver plane)" if w["Nx"][0] == 512 and w["steps"] == 4000
            else f"3D scalar forward with PML ({w['Nx'][0]}^3, radius 4, {w['width']}-cell PML, "
                 f"{w['steps']} steps)",
            "grid": list(w["Nx"]), "space_order": 8, "pml": w["width"], "time_steps": w["steps"],
            "receivers": int(w["sensors"].shape[1]), "precision": "float32",
            "parallelism": f"replicas x{args.gpus}", "l2": "inputs larger than L2 (512 MiB per field)"}


# ------------------------------------------------------------------- our arm
def step_kernel_ms(sim, mat_inputs, steps: int) -> float:
    """Average duration of one march step (its launches: the blocked step with the axis-0
    pml, the pml of axes 1-2, the sources, the refill) over `steps` back-to-back steps on
    the stream they run on, by CUDA events."""
    import torch

    from cuwave_b200 import _native as nat
    from cuwave_b200.wave import forward_ops, pml_memory, prepare_shot

    dev = torch.device("cuda")
    indicator, position, signal = mat_inputs
    mat = sim.build_materials(indicator.clone())
    shot = prepare_shot(sim, mat, position, signal)
    U = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    memory = pml_memory(sim, 3, dev)
    ops = forward_ops(sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
                      nat.level(U, add=0, period=2), shot, memory)
    assert len(ops) == 1 and ops[0].kind == nat.OP_STEP
    plan = sim.plan()
    plan.march(ops, 0, 8)
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    plan.march(ops, 8, steps)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def blob_speed(n: int, seed: int = 0) -> np.ndarray:
    """The blob speed model: 1 plus 8 seeded Gaussian blobs (A in [-0.3, 0.3], sigma in
    [10, 40] cells at 512, scaled with the grid)."""
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    c = np.ones((n, n))
    for _ in range(8):
        a, s = rng.uniform(-0.3, 0.3), rng.uniform(10, 40) * n / 512
        cy, cx = rng.uniform(1, n - 1, 2)
        c += a * np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2 * s * s))
    return c


def march_ms(plan, ops, t0: int, steps: int, base: int = 64) -> float:
    """CUDA-event time of one march step of `ops` on the stream they run on: the time of
    `base + steps` steps less that of `base` steps, over `steps`, so the per-call cost of
    a march (capturing and instantiating its step graph, the closing status read) drops
    out; the best of three."""
    import torch

    stream = torch.cuda.current_stream()

    def run(n):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        plan.march(ops, t0, n)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    run(base + steps)
    long = min(run(base + steps) for _ in range(3))
    short = min(run(base) for _ in range(3))
    return (long - short) / steps


def two_d_kernels(peak: float, steps: int = 200) -> dict:
    """The 2D kernels at the 2D forward and sensitivity shapes (512^2 Neumann; 2048^2 with a
    20-cell PML): the forward step and the adjoint step (pml memory, the transposed update
    with the gradients, the pml gather, the adjoint load), each as Gpt-updates/s and its
    algorithmic HBM bytes over its CUDA-event time."""
    import torch

    from cuwave_b200 import AcousticWave, Pml, _native as nat
    from cuwave_b200.sensitivity import _adjoint_ops
    from cuwave_b200.stencils import stable_dt
    from cuwave_b200.wave import flatten_indices, forward_ops, pml_memory, prepare_shot

    dev = torch.device("cuda")
    out = {}
    for name, n, width in (("forward_2d_512", 512, 0), ("sensitivity_2d_2048", 2048, 20)):
        c = blob_speed(n)
        kappa2 = 0.25
        dt = 0.5 * stable_dt((1.0, 1.0), float(c.max()), 8, "optimized")
        N = steps + 64 + 8  # march_ms's two marches reach step 64 + steps
        sim = AcousticWave(Nx=(n, n), dx=(1.0, 1.0), N=N, dt=dt, precision="float32", space_order=8,
                           pml=Pml(width=width, wavespeed=float(c.max())) if width else None,
                           rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=kappa2)
        ind = torch.zeros(sim.Nx_padded, dtype=torch.float32, device=dev)
        ind[:n, :n] = torch.as_tensor((1.0 / c**2 - 1.0) / (1.0 / kappa2 - 1.0), device=dev)
        mat = sim.build_materials(ind)
        signal = torch.zeros((N, 1), dtype=torch.float32, device=dev)
        shot = prepare_shot(sim, mat, torch.tensor([[n // 2], [n // 2]], device=dev), signal)
        interior = (n - 2) ** 2
        slab = 2 * 2 * width * (n - 2) if width else 0
        U = torch.zeros((2, *sim.Nx_padded), dtype=torch.float32, device=dev)
        ops = forward_ops(sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
                          nat.level(U, add=0, period=2), shot, pml_memory(sim, 3, dev))
        plan = sim.plan()
        ms = march_ms(plan, ops, 0, steps)
        fwd_bytes = 16 * interior + 24 * slab
        entry = {"forward_gpts": interior / (ms / 1e3) / 1e9, "forward_ms_per_step": ms,
                 "forward_roofline_frac": fwd_bytes / (ms / 1e3) / 1e9 / peak}
        if width:
            V = torch.zeros((N + 2, *sim.Nx_padded), dtype=torch.float32, device=dev)
            P = torch.zeros((2, *sim.Nx_padded), dtype=torch.float32, device=dev)
            sensors = torch.stack([torch.full((256,), 50), torch.linspace(30, n - 31, 256).round().long()]).int().to(dev)
            lin = flatten_indices(sim, sensors)
            adj_signal = torch.zeros((N, 256), dtype=torch.float32, device=dev)
            grads = sim.gradient_fields(mat)
            aops = _adjoint_ops(sim, mat, P, pml_memory(sim, 5, dev), u_level=nat.level(V, mul=-1, add=N + 1),
                                grads=grads, load=(lin, adj_signal, sim.excitation_weights(mat, lin)))
            ams = march_ms(plan, aops, 0, steps)
            adj_bytes = 32 * interior + 44 * slab
            entry.update({"adjoint_gpts": interior / (ams / 1e3) / 1e9, "adjoint_ms_per_step": ams,
                          "adjoint_roofline_frac": adj_bytes / (ams / 1e3) / 1e9 / peak})
            del V, P
        out[name] = entry
    return out


def blocked_2d(peak: float, n: int = 8192, steps: int = 64) -> dict:
    """The temporally blocked 2D march against the march of one launch a step, on a grid
    whose fields stream from HBM: n x n, radius 4, Neumann faces, the blob speed model and a
    source at the centre. Per step: its CUDA-event time, Gpt-updates/s and the fraction of
    the measured HBM peak the single-step algorithmic bytes (16 B an update) would need at
    that rate -- above 1 where a pass over HBM serves several steps."""
    import os

    import torch

    from cuwave_b200 import AcousticWave, _native as nat
    from cuwave_b200.stencils import stable_dt
    from cuwave_b200.wave import forward_ops, pml_memory, prepare_shot

    dev = torch.device("cuda")
    c = blob_speed(n)
    kappa2 = 0.25
    dt = 0.5 * stable_dt((1.0, 1.0), float(c.max()), 8, "optimized")
    N = 2 * (steps + 64) + 8
    interior = (n - 2) ** 2
    out = {"grid": [n, n], "space_order": 8}
    for name, mode in (("single", "0"), ("blocked", "2")):
        os.environ["CWB_TBLOCK"] = mode
        try:
            sim = AcousticWave(Nx=(n, n), dx=(1.0, 1.0), N=N, dt=dt, precision="float32",
                               space_order=8, rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=kappa2)
            ind = torch.zeros(sim.Nx_padded, dtype=torch.float32, device=dev)
            ind[:n, :n] = torch.as_tensor((1.0 / c**2 - 1.0) / (1.0 / kappa2 - 1.0), device=dev)
            mat = sim.build_materials(ind)
            shot = prepare_shot(sim, mat, torch.tensor([[n // 2], [n // 2]], device=dev),
                                torch.zeros((N, 1), dtype=torch.float32, device=dev))
            U = torch.zeros((2, *sim.Nx_padded), dtype=torch.float32, device=dev)
            ops = forward_ops(sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
                              nat.level(U, add=0, period=2), shot, pml_memory(sim, 3, dev))
            ms = march_ms(sim.plan(), ops, 0, steps)
        finally:
            os.environ.pop("CWB_TBLOCK", None)
        out[name] = {"ms_per_step": ms, "gpts": interior / (ms / 1e3) / 1e9,
                     "roofline_frac": 16 * interior / (ms / 1e3) / 1e9 / peak}
        del U
    return out


def three_d_kernels(peak: float, n: int = 256, steps: int = 100) -> dict:
    """The 3D steps beside the bench job's radius: the forward step for radius 1..8 on an
    n^3 grid with Neumann faces (radius 1..4 on the register-blocked kernel, 5..8 on the
    row kernel), and the fused adjoint step (transposed update with the gradients, the
    pml transpose, the adjoint load) at radius 4 with a 10-cell pml, each as
    Gpt-updates/s and the fraction of the measured HBM peak its algorithmic bytes give."""
    import torch

    from cuwave_b200 import AcousticWave, Pml, _native as nat
    from cuwave_b200.sensitivity import _adjoint_ops
    from cuwave_b200.stencils import stable_dt
    from cuwave_b200.wave import flatten_indices, forward_ops, pml_memory, prepare_shot

    dev = torch.device("cuda")
    rng = np.random.default_rng(5)
    c = 1.0 + 0.5 * rng.random((n, n, n))
    kappa2 = 0.25
    interior = (n - 2) ** 3
    out = {}
    N = steps + 64 + 8
    for R in range(1, 9):
        width = 10 if R == 4 else 0
        dt = 0.5 * stable_dt((1.0,) * 3, float(c.max()), 2 * R, "optimized")
        sim = AcousticWave(Nx=(n, n, n), dx=(1.0,) * 3, N=N, dt=dt, precision="float32",
                           space_order=2 * R, pml=Pml(width=width, wavespeed=float(c.max())) if width else None,
                           rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=kappa2)
        ind = torch.zeros(sim.Nx_padded, dtype=torch.float32, device=dev)
        ind[..., :n] = torch.as_tensor((1.0 / c**2 - 1.0) / (1.0 / kappa2 - 1.0), device=dev)
        mat = sim.build_materials(ind)
        shot = prepare_shot(sim, mat, torch.tensor([[n // 2]] * 3, device=dev),
                            torch.zeros((N, 1), dtype=torch.float32, device=dev))
        U = torch.zeros((2, *sim.Nx_padded), dtype=torch.float32, device=dev)
        ops = forward_ops(sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
                          nat.level(U, add=0, period=2), shot, pml_memory(sim, 3, dev))
        plan = sim.plan()
        ms = march_ms(plan, ops, 0, steps)
        slab = sum(2 * width * (n - 2) ** 2 for _ in range(3))
        fwd_bytes = 16 * interior + 24 * slab
        entry = {"pml": width, "forward_gpts": interior / (ms / 1e3) / 1e9, "forward_ms_per_step": ms,
                 "forward_roofline_frac": fwd_bytes / (ms / 1e3) / 1e9 / peak}
        if R == 4:
            V = torch.zeros((N + 2, *sim.Nx_padded), dtype=torch.float32, device=dev)
            P = torch.zeros((2, *sim.Nx_padded), dtype=torch.float32, device=dev)
            cols = np.linspace(20, n - 21, 64).round().astype(int).tolist()
            sensors = torch.tensor([[20] * 64, cols, [n // 2] * 64], dtype=torch.int32, device=dev)
            lin = flatten_indices(sim, sensors)
            adj_signal = torch.zeros((N, 64), dtype=torch.float32, device=dev)
            aops = _adjoint_ops(sim, mat, P, pml_memory(sim, 5, dev), u_level=nat.level(V, mul=-1, add=N + 1),
                                grads=sim.gradient_fields(mat), load=(lin, adj_signal, sim.excitation_weights(mat, lin)))
            ams = march_ms(plan, aops, 0, steps)
            adj_bytes = 32 * interior + 44 * slab
            entry.update({"adjoint_gpts": interior / (ams / 1e3) / 1e9, "adjoint_ms_per_step": ams,
                          "adjoint_roofline_frac": adj_bytes / (ams / 1e3) / 1e9 / peak})
            del V, P
        out[f"r{R}"] = entry
        del U
    return {"grid": [n, n, n], "kernels": out}


def batch_problems(count: int, steps: int, seed: int = 3):
    """A topology-optimisation population: `count` 2D designs, sides U{256..1536}, space orders
    {4..12}, two-phase speeds {1.0, 0.3} from a thresholded smooth random field, a
    Ricker source at the centre and 64 receivers on a row; `steps` steps each."""
    import torch
    import torch.nn.functional as F

    from cuwave_b200 import AcousticWave, Source, ricker, stable_dt

    rng = np.random.default_rng(seed)
    problems = []
    for _ in range(count):
        side = int(rng.integers(256, 1537))
        order = int(rng.choice([4, 6, 8, 10, 12]))
        noise = torch.as_tensor(rng.standard_normal((1, 1, side, side)), dtype=torch.float32)
        smooth = F.avg_pool2d(noise, 15, stride=1, padding=7)[0, 0].numpy()
        c = np.where(smooth > 0.0, 1.0, 0.3)
        dx = (1.0, 1.0)
        dt = 0.5 * stable_dt(dx, 1.0, order)
        sim = AcousticWave(Nx=(side, side), dx=dx, N=steps, dt=dt, space_order=order,
                           rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=0.09)
        full = np.ones(sim.Nx_padded)
        full[:side, :side] = c
        ind = AcousticWave.indicator_for_speed(full, 0.09).astype(np.float32)
        t = np.arange(steps) * dt
        src = Source(np.array([[side // 2], [side // 2]], np.int32), ricker(t, 1.0, 0.03)[:, None])
        sens = np.stack([np.full(64, side // 4), np.linspace(2, side - 3, 64).astype(int)]).astype(np.int32)
        problems.append((sim, src, ind, sens))
    return problems


def batch_measure(count: int = 64, steps: int = 1500) -> dict:
    """simulate_batch over the design population (batch_problems) against the same simulate calls in turn
    (device time, CUDA events; the second of two runs, the first tunes and loads)."""
    import torch

    from cuwave_b200 import simulate
    from cuwave_b200.batch import simulate_batch

    problems = batch_problems(count, steps)
    updates = sum((p[0].Nx[0] - 2) * (p[0].Nx[1] - 2) * p[0].N for p in problems)
    sims, srcs, inds, sens = (list(x) for x in zip(*problems))
    out = {}
    for rep in range(2):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        simulate_batch(sims, srcs, [i.copy() for i in inds], sens)
        e1.record()
        for sim, src, ind, s in problems:
            simulate(sim, src, ind.copy(), s)
        e2.record()
        torch.cuda.synchronize()
        out = {"problems": count, "steps": steps, "updates": updates,
               "batch_s": e0.elapsed_time(e1) / 1e3, "in_turn_s": e1.elapsed_time(e2) / 1e3}
    out["batch_gpts"] = updates / out["batch_s"] / 1e9
    out["in_turn_gpts"] = updates / out["in_turn_s"] / 1e9
    return out


def sensitivity_e2e(kernels: dict | None, n: int = 2048, steps: int = 300) -> dict:
    """The 2D gradient job end to end through `sensitivity` (forward with its history,
    the traces' misfit, the adjoint with the gradients): the first call (plan, CUDA
    graphs, the history's allocation) and the best of three warm calls, timed with CUDA
    events, against the march kernels alone (the forward and adjoint steps of
    `kernels_2d` at the same grid, times the steps)."""
    import torch

    from cuwave_b200 import Source, simulate
    from cuwave_b200.sensitivity import l2_misfit, sensitivity

    w = sensitivity_workload(n, steps)
    sim = make_sim_2d(w)
    dev = torch.device("cuda")
    src = Source(torch.as_tensor(w["source"], device=dev), torch.as_tensor(w["signal"], device=dev))
    sens = torch.as_tensor(w["sensors"], device=dev)
    _, observed = simulate(sim, src, torch.as_tensor(w["indicator_obs"], device=dev).clone(), sens)
    objective = l2_misfit(observed)
    ind = torch.as_tensor(w["indicator"], device=dev)

    def timed() -> float:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        cost, grads, _, _ = sensitivity(sim, src, ind.clone(), sens, objective)
        b.record()
        torch.cuda.synchronize()
        assert bool(torch.isfinite(grads["mass"]).all()) and np.isfinite(float(cost))
        return a.elapsed_time(b)

    first = timed()
    warm = min(timed() for _ in range(3))
    updates = 2 * steps * (n - 2) ** 2  # forward and adjoint
    out = {"grid": [n, n], "steps": steps, "pml": w["width"], "first_call_ms": first, "warm_ms": warm,
           "gpts": updates / (warm / 1e3) / 1e9}
    entry = (kernels or {}).get("sensitivity_2d_2048")
    if entry and n == 2048:
        kernel_ms = steps * (entry["forward_ms_per_step"] + entry["adjoint_ms_per_step"])
        out.update({"kernels_ms": kernel_ms, "over_kernels": warm / kernel_ms})
    return out


def shots_measure(count: int = 96, steps: int = 2000, n: int = 1024) -> dict:
    """A multi-shot gradient: `count` shots on a shared n^2 grid (blob speeds, radius 4),
    sources evenly spaced along the top, 256 receivers 50 cells down, `steps` steps;
    the summed misfit gradient (a forward with its history and an adjoint per shot),
    the shots side by side on `misfit_gradient`'s lanes and then in turn, wall-clock
    with the device synchronized on both sides, after a warm-up of one shot a lane; the
    two results compared to the bit. Observed data are zero, so the misfit is the
    traces' energy."""
    import torch

    from cuwave_b200 import AcousticWave, ricker
    from cuwave_b200.stencils import stable_dt
    from cuwave_b200.utils import Sensors, misfit_gradient, shots

    c = blob_speed(n)
    kappa2 = 0.25
    dt = 0.5 * stable_dt((1.0, 1.0), float(c.max()), 8, "optimized")
    sim = AcousticWave(Nx=(n, n), dx=(1.0, 1.0), N=steps, dt=dt, precision="float32",
                       space_order=8, rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=kappa2)
    ind = np.zeros(sim.Nx_padded, np.float32)
    ind[:n, :n] = (1.0 / c**2 - 1.0) / (1.0 / kappa2 - 1.0)
    # about 20 points a wavelength at the peak frequency
    signal = ricker(np.arange(steps) * dt, 1.0, float(c.min()) / 20.0)
    coords = np.stack([np.full(count, 10.0), np.linspace(20.0, n - 21.0, count)], axis=1)
    sources = shots(sim, coords, signal)
    sensors = Sensors(sim, np.stack([np.full(256, 50.0), np.linspace(20.0, n - 21.0, 256)], axis=1))
    observed = [torch.zeros((steps, 256), dtype=torch.float32, device="cuda")] * count
    from cuwave_b200.utils import _lanes
    from cuwave_b200.sensitivity import sensitivity

    lanes = _lanes(sim, count, sensitivity)
    misfit_gradient(sim, sources[:lanes], ind, sensors, observed[:lanes])  # plans, graphs

    def timed(k):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = misfit_gradient(sim, sources, ind, sensors, observed, lanes=k)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, out

    seconds, (cost, gradient) = timed(lanes)
    turn_s, (cost1, gradient1) = timed(1)
    same = bool(cost == cost1 and torch.equal(gradient, gradient1))
    updates = 2 * count * steps * (n - 2) ** 2  # forward and adjoint
    return {"shots": count, "steps": steps, "grid": [n, n], "space_order": 8,
            "receivers": 256, "lanes": lanes, "seconds": seconds, "in_turn_s": turn_s,
            "shots_per_s": count / seconds, "gpts": updates / seconds / 1e9,
            "over_in_turn": turn_s / seconds, "equal_to_in_turn": same,
            "finite": bool(np.isfinite(cost))}


def learned_measure(coarse_nodes: int = 256, coarse_steps: int = 600) -> dict:
    """The learned coarse-grid form at a reduced size: the corrector trained on pairs the plain solver makes,
    then on held-out speed models the fine solve, the plain coarse solve and the corrected
    coarse solve timed (CUDA events) and their receiver traces compared with the fine
    ones (relative L2)."""
    import torch

    from cuwave_b200 import corrector as cr

    pair = cr.grid_pair(coarse_nodes, 1.0, 2.0, coarse_steps)
    rng = np.random.default_rng(0)
    inputs, targets = cr.training_pairs(pair, rng, shots=12, windows=12)
    net = cr.Corrector(seed=1)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    losses = cr.train(net, inputs, targets, steps=800, batch=8, lr=5e-4)
    t1.record()
    torch.cuda.synchronize()
    held = np.random.default_rng(99)
    rows = []
    Nc = coarse_nodes
    for _ in range(3):
        c = cr.speed_field(held, Nc)
        pos = held.integers(Nc // 4, 3 * Nc // 4, size=2)
        fsrc, csrc = cr.shot_sources(pair, pos)
        cs = np.stack([np.full(16, Nc // 5), np.linspace(3, Nc - 4, 16).astype(int)]).astype(np.int32)
        fs = (2 * cs - 1).astype(np.int32)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        fine = cr.fine_traces(pair, c, fsrc, fs)
        ev[1].record()
        plain, _ = cr.corrected_traces(pair, None, c, csrc, cs)
        ev[2].record()
        corr, est = cr.corrected_traces(pair, net, c, csrc, cs)
        ev[3].record()
        torch.cuda.synchronize()
        n = min(fine.shape[0], plain.shape[0])
        err = lambda a: float((a[:n] - fine[:n]).norm() / fine[:n].norm())  # noqa: E731
        rows.append({"fine_ms": ev[0].elapsed_time(ev[1]), "coarse_ms": ev[1].elapsed_time(ev[2]),
                     "corrected_ms": ev[2].elapsed_time(ev[3]), "coarse_error": err(plain),
                     "corrected_error": err(corr), "estimate": est})
    return {"coarse_grid": [Nc, Nc], "fine_grid": list(pair.fine.Nx), "coarse_steps": coarse_steps,
            "fine_steps": pair.fine.N, "train_s": t0.elapsed_time(t1) / 1e3,
            "train_loss_first": float(np.mean(losses[:5])), "train_loss_last": float(np.mean(losses[-50:])),
            "held_out": rows}


def run_ours(args) -> int:
    import torch
    import torch.distributed as dist

    from cuwave_b200 import Source, _native as nat, simulate

    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    w = workload(args.size, args.nt, args.pml)
    sim = make_sim(w)
    dev = torch.device("cuda", local)
    indicator = torch.as_tensor(w["indicator"], device=dev)
    position = torch.as_tensor(w["source"], device=dev)
    signal = torch.as_tensor(w["signal"], device=dev)
    sensors = torch.as_tensor(w["sensors"], device=dev)
    source = Source(position, signal)

    def job():
        return simulate(sim, source, indicator.clone(), sensors)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t)

    for _ in range(args.warmup):
        job()
    barrier()
    clocks = ClockSampler(local)
    launches0 = nat.launches()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        field, traces = job()
    e1.record(stream)
    barrier()
    clock = clocks.stop()
    launches = nat.launches() - launches0
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    updates = interior_updates(w) * w["steps"]
    value = world * updates / (ms / 1e3) / 1e9

    # e2e: the public call from pinned host buffers, results copied back, every step
    host_ind = torch.as_tensor(w["indicator"]).pin_memory()
    host_pos = torch.as_tensor(w["source"]).pin_memory()
    host_sig = torch.as_tensor(w["signal"]).pin_memory()
    host_sens = torch.as_tensor(w["sensors"]).pin_memory()
    out_field = torch.empty(tuple(w["Nx"]), dtype=torch.float32).pin_memory()
    out_traces = torch.empty((w["steps"], w["sensors"].shape[1]), dtype=torch.float32).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in (host_ind, host_pos, host_sig, host_sens))
    d2h = sum(t.numel() * t.element_size() for t in (out_field, out_traces))

    def e2e_job():
        f, um = simulate(sim, Source(host_pos, host_sig), host_ind, host_sens)
        out_field.copy_(f, non_blocking=True)
        out_traces.copy_(um, non_blocking=True)

    e2e_job()
    barrier()
    e2e_steps = max(1, min(args.steps, 10))
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_job()
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps)
    e2e_value = world * updates / (e2e_ms / 1e3) / 1e9

    # the dominant kernel against the HBM roofline
    kernel_ms = step_kernel_ms(sim, (indicator, position, signal), args.kernel_steps)
    kernel_ms = max_over_ranks(kernel_ms)
    bytes_per_launch = algorithmic_bytes(w)
    achieved = bytes_per_launch / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = hbm_peak()
    traffic = profile_traffic(w)
    kernels_2d = two_d_kernels(peak) if args.size == 512 and not args.no_2d and world == 1 else None
    sens_2d = sensitivity_e2e(kernels_2d) if kernels_2d is not None else None
    kernels_3d = three_d_kernels(peak) if args.size == 512 and not args.no_3d and world == 1 else None
    blocked = blocked_2d(peak) if args.size == 512 and not args.no_2d and world == 1 else None
    batch = batch_measure() if args.size == 512 and not args.no_batch and world == 1 else None
    shots_2d = shots_measure() if args.size == 512 and not args.no_batch and world == 1 else None
    learned = learned_measure() if args.size == 512 and args.learned and world == 1 else None

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    baseline, parity = None, None
    if not args.no_cpu:
        baseline, ref_field, ref_traces = cpu_baseline(w, args.cpu_sample)
        if ref_field is not None:
            parity = sample_parity(sim, w, args.cpu_sample, ref_field, ref_traces)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered model)",
        "config": config_line(w, args),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "kernel": step_kernel_name(),
                     "kernel_ms": kernel_ms, "algorithmic_bytes_per_launch": bytes_per_launch},
        "cpu_baseline": baseline,
        "parity": parity,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "gpu_launches": launches,
        "clocks": clock,
        "kernel_updates_per_s": interior_updates(w) / (kernel_ms / 1e3) / 1e9,
        "kernels_2d": kernels_2d,
        "sensitivity_2d": sens_2d,
        "kernels_3d": kernels_3d,
        "blocked_2d": blocked,
        "batch_2d": batch,
        "shots_2d": shots_2d,
        "learned": learned,
    }
    print(json.dumps(line))
    return 0


def step_kernel_name() -> str:
    if os.environ.get("CWB_STEP3D", "1") != "0" and os.environ.get("CWB_NO_TMA", "0") == "0":
        step = ("step3d_flow_kernel<float,4>" if os.environ.get("CWB_FLOW3D", "1") != "0"
                else "step3d_kernel<float,4,uniform>")
        tail = ("refill3d_kernel (refill, sources, receivers)" if os.environ.get("CWB_FOLD3D", "1") != "0"
                else "excite_kernel + refill3d_kernel + record_kernel")
        return (f"one march step: {step} (fd + axis-0 pml) + "
                f"pml_axis1_kernel + pml_axis2_kernel (axes 1-2) + {tail}")
    return "step_tma_kernel<float,3,4,uniform> (row step: fd + pml + sources + refill)"


def hbm_peak() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


def profile_traffic(w: dict):
    """DRAM bytes of one march step (all its launches) from the committed ncu summary
    (profiles/traffic.json, captured on a smaller grid): each kernel's bytes per unit
    (interior node, slab node of axes 1-2, face node) scaled to this workload, or None
    when no capture was summarised."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return None
    data = json.loads(path.read_text())["kernels"]
    n, wd = w["Nx"][0] - 2, w["width"]
    units = {"interior nodes": n**3, "slab nodes of axes 1 and 2": n * 2 * wd * n + n * (n - 2 * wd) * 2 * wd,
             "slab nodes of axis 1": n * 2 * wd * n, "slab nodes of axis 2": n * n * 2 * wd,
             "face nodes": 6 * n * n, "face nodes of axes 0 and 1": 4 * n * n,
             "sources": w["source"].shape[1]}
    total = 0.0
    for entry in data.values():
        if entry["unit"] not in units:
            return None
        total += entry["bytes_per_unit"] * units[entry["unit"]]
    return total


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--size", type=int, default=512, help="grid nodes per axis (ghosts included)")
    parser.add_argument("--nt", type=int, default=4000, help="time steps of one job")
    parser.add_argument("--pml", type=int, default=20, help="pml width in cells (0: none)")
    parser.add_argument("--kernel-steps", type=int, default=400)
    parser.add_argument("--cpu-sample", type=int, default=6, help="time steps the CPU baseline runs")
    parser.add_argument("--ref-sample", type=int, default=3, help="time steps per reference bench step")
    parser.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    parser.add_argument("--no-2d", action="store_true", help="skip the 2D kernel measurements")
    parser.add_argument("--no-3d", action="store_true", help="skip the 3D kernel measurements beside the job's")
    parser.add_argument("--no-batch", action="store_true", help="skip the batched 2D march")
    parser.add_argument("--learned", action="store_true",
                        help="also train and time the learned corrector (not yet a gain)")
    parser.add_argument("--case", choices=("kernels_2d", "kernels_3d", "blocked_2d"),
                        help="run one of the kernel measurements alone and print it (profiling)")
    parser.add_argument("--case-size", type=int, default=None, help="grid nodes per axis of --case")
    args = parser.parse_args(argv)
    if args.case:
        import torch

        torch.cuda.set_device(0)
        peak = hbm_peak()[0]
        if args.case == "kernels_2d":
            out = two_d_kernels(peak)
        elif args.case == "kernels_3d":
            out = three_d_kernels(peak, n=args.case_size or 256)
        else:
            out = blocked_2d(peak, n=args.case_size or 8192)
        print(json.dumps(out))
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
