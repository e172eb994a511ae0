"""Adjoint sensitivities: `sensitivity`, `reconstruction_sensitivity`,
`superposition_sensitivity`, `spectral_sensitivity`, `source_sensitivity`.

Same arguments and returns as cuwave `sensitivity.py` (384-497, 500-750, 753-893,
896-1051, 1054-1111):
`(cost, {"mass": dJ/dm, "stiff": dJ/dk}, traces, info)` with the gradients over the
padded grid, cell-weighted and zeroed in a pml layer, or `(cost, dJ/dsignal, traces,
info)` for the source. The adjoint marches run in the native library: the transposed
step with the gradients fused in (CWB_OP_ADJOINT), the pml transpose (CWB_OP_PML_AUX and
the gather inside the step) and the adjoint load (CWB_OP_LOAD).
"""

from __future__ import annotations

import itertools
import math
import warnings
from collections.abc import Callable
from dataclasses import replace

import numpy as np
import torch

from . import _native as nat
from .boundary import pml_nodes
from .wave import (
    BFLOAT16,
    Simulation,
    Source,
    as_device,
    as_position,
    device,
    flatten_indices,
    forward_ops,
    grid_rows,
    narrow,
    pml_memory,
    prepare_shot,
    require_off_held_walls,
    simulate,
)

# what `strip_dtype` stores the strip as, per (strip_dtype, precision) (cuwave sensitivity.py:54-58)
STRIP_DTYPES = {
    ("float32", "float64"): torch.float32,
    ("bfloat16", "float32"): BFLOAT16,
    ("bfloat16", "float64"): BFLOAT16,
}
# round-off growth past which a damped node is recorded rather than run backwards
REVERSIBLE_GROWTH = {"float32": 1e2, "float64": 1e6}
# lines the adjoint up with the reconstructed forward triplet (cuwave sensitivity.py:45)
ADJOINT_DELAY = 1
# cancellation past which B(w, w) - B(u, u) has eaten too much of the mantissa to trust
CANCELLATION_LIMIT = {"float32": 1e5, "float64": 1e12}
# share of the spectrum the last period still adds, past which the run stopped short
DECAY_LIMIT = 1e-2
# dcost/dtraces off the sinusoids at `frequencies` by more than this is not spectral
FIT_LIMIT = {"float32": 1e-4, "float64": 1e-10}
PULSE_PERIODS = 1.0  # spread of the adjoint pulse envelope, in periods


def l2_misfit(observed) -> Callable:
    """Objective factory: J = 1/2 sum (traces - observed)^2 and its derivative (cuwave sensitivity.py:93-100)."""

    def objective(traces):
        residual = traces - as_device(observed, traces.dtype)
        return 0.5 * float(torch.sum(residual**2)), residual

    return objective


def windowed_misfit(observed, window) -> Callable:
    """`l2_misfit` restricted to a time window (cuwave sensitivity.py:68-84)."""

    def objective(traces):
        w = as_device(window, traces.dtype)
        residual = w * (traces - as_device(observed, traces.dtype))
        return 0.5 * float(torch.sum(residual**2)), w * residual

    return objective


def require_interior(sim: Simulation, position, what: str) -> None:
    """Raise if a node of `position` sits on a ghost (cuwave sensitivity.py:103-118)."""
    rows = grid_rows(sim, as_position(sim, position))
    if rows.numel() == 0:
        return
    lo = int(rows.min())
    if lo < 1:
        raise ValueError(f"{what} on a ghost node: index {lo} < 1")
    for d in range(sim.ndim):
        hi = int(rows[d].max())
        if hi > sim.Nx[d] - 2:
            raise ValueError(
                f"{what} on a ghost node: axis {d} index {hi} exceeds Nx[{d}] - 2 = {sim.Nx[d] - 2}"
            )


def require_full_domain(sim: Simulation) -> None:
    """Raise for a masked domain: the gradient kernels grade no wall (cuwave sensitivity.py:121-127)."""
    if sim.masked:
        raise NotImplementedError(
            "the gradient kernels read every cell at the full radius, where a domain closes "
            "some; unset domain, or use source_sensitivity, which needs none"
        )


def frozen(sim: Simulation, grads: dict) -> dict:
    """`grads` zeroed in the pml layer, assigned so a NaN cannot survive (cuwave sensitivity.py:198-205)."""
    if sim.pml is not None:
        layer = torch.as_tensor(pml_nodes(sim), device=next(iter(grads.values())).device)
        for f in grads.values():
            f[layer] = 0.0
    return grads


def adjoint_signal(sim: Simulation, dphi, sensors, scale: float = 1.0, delay: int = 0):
    """dphi reversed in time over W and the source factor (cuwave sensitivity.py:272-292)."""
    sensors = as_position(sim, sensors)
    signal = as_device(dphi, sim.dtype).flip(0) / sim.adjoint_weights(sensors)
    if delay:
        signal = torch.cat((signal[delay:], torch.zeros_like(signal[:delay])))
    return (torch.tensor(scale, dtype=sim.dtype, device=signal.device) * signal).contiguous()


def _objective(objective, um):
    cost, dphi = objective(um)
    return float(cost), dphi


def _adjoint_ops(sim, mat, P, eta, *, u_level=None, grads=None, load=None, probe=None):
    """One adjoint step lambda^n in P[m % 2] from P[(m + 1) % 2]: pml memory, the
    transposed update (gradients fused against `u_level` when `grads`), the load, and a
    probe of lambda after the load."""
    material = sim.material(mat)
    l0 = nat.level(P, add=0, period=2)
    l1 = nat.level(P, add=1, period=2)
    ops = []
    flags = 0
    if sim.pml is not None:
        ops.append(nat.op(nat.OP_PML_AUX, a=l1, mat=material, memory=eta))
        flags |= nat.PML
    fields = dict(a=l0, b=l1, mat=material, memory=eta, scale=sim.adjoint_mass_factor())
    if grads is not None:
        flags |= nat.GRAD
        fields.update(c=u_level, g_mass=grads["mass"], g_stiff=grads["stiff"])
    ops.append(nat.op(nat.OP_ADJOINT, flags=flags, **fields))
    if load is not None:
        lin, signal, weight = load
        pts = nat.points(lin, signal, weight=weight)
        if grads is not None:
            ops.append(nat.op(nat.OP_LOAD, a=l0, c=u_level, points=pts, g_mass=grads["mass"],
                              scale=sim.adjoint_mass_factor()))
        else:
            ops.append(nat.op(nat.OP_EXCITE, a=l0, points=pts))
    if probe is not None:
        lin, record = probe
        ops.append(nat.op(nat.OP_RECORD, a=l0, points=nat.points(lin, record)))
    return ops


def sensitivity(sim: Simulation, source: Source, indicator, sensors, objective: Callable,
                *, _mat: dict | None = None, _probe: bool = False):
    """Cost and d(cost)/d(mass, stiff) with the forward history stored (cuwave sensitivity.py:384-497).

    The forward march writes every level into an (N + 2)-level history V, V[t + 2] = u^t;
    the adjoint march steps lambda with the gradients fused against V reversed.
    (`_mat` replaces the materials built from `indicator`; `_probe` also returns
    d(cost)/d(source.signal) in info["source"], from the same adjoint march.)
    """
    require_interior(sim, sensors, "sensor")
    require_interior(sim, source.position, "source")
    require_full_domain(sim)
    dev = device()
    mat = sim.build_materials(indicator) if _mat is None else _mat
    shot = prepare_shot(sim, mat, source.position, source.signal)
    require_off_held_walls(sim, shot.position)
    plan = sim.plan()
    N = sim.N

    # ---------------------------------------------------------------- forward pass
    V = torch.zeros((N + 2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    memory = pml_memory(sim, 3, dev)
    ops = forward_ops(sim, mat, nat.level(V, add=0), nat.level(V, add=1), nat.level(V, add=2),
                      shot, memory)
    plan.march(ops, 0, N)
    del memory
    sensor_lin = flatten_indices(sim, sensors)
    # column-major, as numpy lays out the reference's V[2:][:, lin]: a sum over a
    # reshaped record then adds in the same order
    um = V[2:].reshape(N, -1).t().index_select(0, sensor_lin.long()).t()
    cost, dphi = _objective(objective, um)

    # --------------------------------------------------------------- backward pass
    signal = adjoint_signal(sim, dphi, sensors)
    weight = sim.excitation_weights(mat, sensor_lin)
    grads = sim.gradient_fields(mat)
    P = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    eta = pml_memory(sim, 5, dev)
    # adjoint step m pairs lambda^n, n = N - 1 - m, with u^n = V[N + 1 - m]
    u_level = nat.level(V, mul=-1, add=N + 1)
    probe = lam = None
    if _probe:
        lam = torch.zeros((N, shot.lin.numel()), dtype=sim.dtype, device=dev)
        probe = (shot.lin, lam)
    ops = _adjoint_ops(sim, mat, P, eta, u_level=u_level, grads=grads,
                       load=(sensor_lin, signal, weight), probe=probe)
    plan.march(ops, 0, N)
    info = {}
    if _probe:
        info["source"] = (lam.flip(0) * sim.adjoint_weights(shot.position)).contiguous()
    return cost, frozen(sim, sim.finalize_gradients(grads)), um, info


def source_sensitivity(sim: Simulation, source: Source, indicator, sensors, objective: Callable):
    """Cost and d(cost)/d(source.signal) (cuwave sensitivity.py:1054-1111).

    No forward field is stored: the gradient is lambda at the sources, reversed, times
    the adjoint weights.
    """
    require_interior(sim, sensors, "sensor")
    require_interior(sim, source.position, "source")
    dev = device()
    um = simulate(sim, source, indicator, sensors)[1]
    cost, dphi = _objective(objective, um)
    mat = sim.build_materials(indicator)
    plan = sim.plan()
    signal = adjoint_signal(sim, dphi, sensors)
    sensor_lin = flatten_indices(sim, sensors)
    weight = sim.excitation_weights(mat, sensor_lin)
    position = as_position(sim, source.position)
    source_lin = flatten_indices(sim, position)
    P = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    eta = pml_memory(sim, 5, dev)
    lam = torch.zeros((sim.N, source_lin.numel()), dtype=sim.dtype, device=dev)
    if sim.masked:
        # a masked domain steps its adjoint with the graded forward step itself, its own
        # transpose (cuwave scalar.py:322-324), the ghosts refilled as the walls read them
        l0 = nat.level(P, add=0, period=2)
        ops = [
            nat.op(nat.OP_STEP, a=l0, b=nat.level(P, add=1, period=2), c=l0,
                   mat=sim.material(mat)),
            nat.op(nat.OP_EXCITE, a=l0, points=nat.points(sensor_lin, signal, weight=weight)),
            nat.op(nat.OP_REFILL, a=l0),
            nat.op(nat.OP_RECORD, a=l0, points=nat.points(source_lin, lam)),
        ]
    else:
        ops = _adjoint_ops(sim, mat, P, eta, load=(sensor_lin, signal, weight),
                           probe=(source_lin, lam))
    plan.march(ops, 0, sim.N)
    gradient = lam.flip(0) * sim.adjoint_weights(position)
    return cost, gradient.contiguous(), um, {}


# ------------------------------------------------------------------- superposition
def require_lossless(sim: Simulation) -> None:
    """Raise for a damping field or a pml: time reversal needs a lossless step (cuwave sensitivity.py:130-136)."""
    if sim.damping is not None or sim.pml is not None:
        raise NotImplementedError(
            "superposition_sensitivity rebuilds the forward field by running it backwards, "
            "which only a lossless operator allows; use sensitivity"
        )


def _accumulated(accs: dict) -> float:
    """The norm over every accumulator (cuwave sensitivity.py:85-88)."""
    return math.sqrt(sum(float(torch.linalg.vector_norm(f)) ** 2 for f in accs.values()))


def _density_factors(sim: Simulation, sign: float) -> tuple[float, float]:
    """(mass, stiffness) density factors of the superposed step, rounded to the
    simulation's dtype (cuwave scalar.py:813-838)."""
    factors = sim.step_factors()
    ratios = [-sign / (2.0 * d) ** 2 / float(f) for d, f in zip(sim.dx, factors)]
    if not np.allclose(ratios, ratios[0]):
        raise ValueError(f"step factors {factors} are not proportional to 1 / dx**2")
    return (float(sim.np_dtype(sign / (2.0 * sim.dt) ** 2)), float(sim.np_dtype(ratios[0])))


def superposition_sensitivity(sim: Simulation, source: Source, indicator, sensors,
                              objective: Callable, scale: float = 1.0):
    """Cost and gradients as `sensitivity`, in three field slots instead of N + 2
    (cuwave sensitivity.py:753-893).

    The gradient densities are bilinear in the forward and adjoint fields, so the cross
    term is read off B(u + k lambda) - B(u): the forward march subtracts B(u, u) as it
    steps (CWB_OP_SUPERPOSED), then the lossless field runs back in time from its last
    two levels carrying w = u + k lambda (the source reversed, the adjoint load scaled
    by k and one step late) and adds B(w, w); the Frechet kernel (CWB_OP_FRECHET) closes
    each pass with its last triplet's mass density. The difference over 2k is the
    gradient, cell weighted. `scale` is k: the cancellation it leaves is returned in
    info["cancellation"], with a warning past what the precision can carry.
    """
    require_lossless(sim)
    require_interior(sim, sensors, "sensor")
    require_interior(sim, source.position, "source")
    require_full_domain(sim)
    dev = device()
    mat = sim.build_materials(indicator)
    shot = prepare_shot(sim, mat, source.position, source.signal)
    require_off_held_walls(sim, shot.position)
    plan = sim.plan()
    N = sim.N
    material = sim.material(mat)
    accs = sim.gradient_fields(mat)
    U = torch.zeros((3, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    sensor_lin = flatten_indices(sim, sensors)
    um = torch.zeros((N, sensor_lin.numel()), dtype=sim.dtype, device=dev)
    zero = (0.0, 0.0, 0.0)

    def frechet(a, b, c, ft):
        return nat.op(nat.OP_FRECHET, a=nat.level(U, mul=0, add=a), b=nat.level(U, mul=0, add=b),
                      c=nat.level(U, mul=0, add=c), g_mass=accs["mass"],
                      g_stiff=accs["stiff"], scale=ft, factors=zero)

    # ---------------------------------------------------------------- forward pass
    # step t: U[t % 3], U[(t + 1) % 3] -> U[(t + 2) % 3], the mass density one triplet late
    ft, fs = _density_factors(sim, -1.0)
    a = nat.level(U, add=0, period=3)
    b = nat.level(U, add=1, period=3)
    c = nat.level(U, add=2, period=3)
    ops = [nat.op(nat.OP_SUPERPOSED, a=a, b=b, c=c, mat=material, g_mass=accs["mass"],
                  g_stiff=accs["stiff"], scale=ft, factors=(fs, 0.0, 0.0))]
    src = shot.points()
    if src.num:
        ops.append(nat.op(nat.OP_EXCITE, a=c, points=src))
    ops.append(nat.op(nat.OP_REFILL, a=c))
    if sensor_lin.numel():
        ops.append(nat.op(nat.OP_RECORD, a=c, points=nat.points(sensor_lin, um)))
    plan.march(ops, 0, N)
    t = N - 1
    plan.march([frechet(t % 3, (t + 1) % 3, (t + 2) % 3, ft)], 0, 1, graph=False)
    cost, dphi = _objective(objective, um)

    # ----------------------------------------------------------- adjoint excitation
    before = _accumulated(accs)
    position = torch.cat((as_position(sim, sensors), shot.position), dim=1)
    lin = flatten_indices(sim, position)
    signal = torch.cat(
        (adjoint_signal(sim, dphi, sensors, scale, ADJOINT_DELAY), shot.signal[:N].flip(0)),
        dim=1,
    ).contiguous()
    weight = sim.excitation_weights(mat, lin)
    load = nat.points(lin, signal, weight=weight)

    # --------------------------------------------------------------- backward pass
    # step t: U[(N + 1 - t) % 3], U[(N - t) % 3] -> U[(N + 2 - t) % 3], from u^(N-1), u^(N-2)
    ft, fs = _density_factors(sim, 1.0)

    def backward_ops(mass_factor):
        a = nat.level(U, mul=-1, add=N + 1, period=3)
        b = nat.level(U, mul=-1, add=N, period=3)
        c = nat.level(U, mul=-1, add=N + 2, period=3)
        return [
            nat.op(nat.OP_SUPERPOSED, a=a, b=b, c=c, mat=material, g_mass=accs["mass"],
                   g_stiff=accs["stiff"], scale=mass_factor, factors=(fs, 0.0, 0.0)),
            nat.op(nat.OP_EXCITE, a=c, points=load),
            nat.op(nat.OP_REFILL, a=c),
        ]

    # the first triplet before is the forward's last, already counted
    plan.march(backward_ops(0.0), 0, 1, graph=False)
    plan.march(backward_ops(ft), 1, N - 1)
    plan.march([frechet(2, 1, 0, ft)], 0, 1, graph=False)

    after = _accumulated(accs)
    cancellation = before / after if after > 0.0 else float("inf")
    limit = CANCELLATION_LIMIT[sim.precision]
    if cancellation > limit:
        warnings.warn(
            f"superposition scale={scale:g} leaves a cancellation of {cancellation:.1e} in "
            f"{sim.precision}, past the usable {limit:.0e}: the gradient is largely "
            f"round-off. Raise scale by about {cancellation / limit:.0e}.",
            RuntimeWarning,
            stacklevel=2,
        )
    norm = float(sim.np_dtype(1.0 / (2.0 * scale)))
    accs = sim.finalize_gradients(accs)
    for f in accs.values():
        f *= norm
    return cost, accs, um, {"scale": scale, "cancellation": cancellation}


# ------------------------------------------------------------------------ spectral
def phase_table(sim: Simulation, frequencies) -> np.ndarray:
    """(N, 2F) host table of cos(omega t) and -sin(omega t), interleaved per frequency,
    built in float64 (cuwave sensitivity.py:295-303)."""
    t = np.arange(sim.N, dtype=np.float64) * sim.dt
    phase = 2.0 * np.pi * t[:, None] * np.asarray(frequencies, np.float64)[None, :]
    table = np.empty((sim.N, 2 * phase.shape[1]))
    table[:, 0::2] = np.cos(phase)
    table[:, 1::2] = -np.sin(phase)
    return table


def spectral_load(sim: Simulation, dphi, table: np.ndarray) -> tuple[np.ndarray, float]:
    """The complex load alpha + i beta per frequency with dphi = sum alpha cos + beta sin,
    by least squares on the host, and the fit's relative residual (cuwave
    sensitivity.py:306-321)."""
    basis = np.empty_like(table)
    basis[:, 0::2], basis[:, 1::2] = table[:, 0::2], -table[:, 1::2]
    if isinstance(dphi, torch.Tensor):
        dphi = dphi.detach().cpu().numpy()
    target = np.asarray(dphi).astype(np.float64)
    coef = np.linalg.lstsq(basis, target, rcond=None)[0]
    norm = float(np.linalg.norm(target))
    fit = float(np.linalg.norm(target - basis @ coef)) / norm if norm > 0.0 else 0.0
    return coef[0::2] + 1j * coef[1::2], fit


def spectral_pulse(sim: Simulation, frequency: float, load: np.ndarray) -> np.ndarray:
    """(N, num) Gaussian-windowed pulses whose DTFT at `frequency` is `load`
    (cuwave sensitivity.py:324-342)."""
    sigma = PULSE_PERIODS / frequency
    t = np.arange(sim.N, dtype=np.float64) * sim.dt
    if 8.0 * sigma > t[-1]:
        raise ValueError(
            f"the adjoint pulse spans {8.0 * sigma:.3g}, longer than the run {t[-1]:.3g}"
        )
    envelope = np.exp(-0.5 * ((t - 4.0 * sigma) / sigma) ** 2)
    omega = 2.0 * np.pi * frequency
    carriers = envelope * np.stack((np.cos(omega * t), np.sin(omega * t)))
    spectra_ = carriers @ np.exp(-1j * omega * t)
    system = np.array([spectra_.real, spectra_.imag])
    amplitudes = np.linalg.solve(system, np.stack((load.real, load.imag)))
    return carriers.T @ amplitudes


def settled(sim: Simulation, spectrum: np.ndarray, last: np.ndarray, frequency: float):
    """The DFT continued past step N as the constant the run settled to, its geometric
    tail summed in closed form (cuwave sensitivity.py:345-354)."""
    z = np.exp(-2j * np.pi * frequency * sim.dt)
    return spectrum + last * (z**sim.N / (1.0 - z))


def spectra(sim: Simulation, acc: np.ndarray, last: np.ndarray, frequency: float, steps: int):
    """One frequency's settled DFT from its (4, num) accumulator (whole run, then the last
    `steps`), and the share of it the last steps added, the settled constant taken out
    (cuwave sensitivity.py:357-380). Host arithmetic in numpy complex128."""
    whole = acc[0].astype(np.complex128) + 1j * acc[1]
    tail = acc[2].astype(np.complex128) + 1j * acc[3]
    z = np.exp(-2j * np.pi * frequency * sim.dt)
    tail = tail - last * complex(np.sum(z ** np.arange(sim.N - steps, sim.N)))
    norm = float(np.linalg.norm(whole))
    share = float(np.linalg.norm(tail)) / norm if norm > 0.0 else 0.0
    return settled(sim, whole, last, frequency), share


def _dilated(sim: Simulation, region: torch.Tensor, reach: int) -> torch.Tensor:
    """`region` grown by `reach` nodes in the max norm (a square structuring element
    applied `reach` times), over the padded grid."""
    x = region.to(torch.float32)[None, None]
    pool = torch.nn.functional.max_pool2d if sim.ndim == 2 else torch.nn.functional.max_pool3d
    return pool(x, kernel_size=2 * reach + 1, stride=1, padding=reach)[0, 0] > 0


def spectral_sensitivity(sim: Simulation, source: Source, indicator, sensors,
                         objective: Callable, frequencies, region=None):
    """Cost and gradients as `sensitivity` for a cost read off the record's spectrum
    (cuwave sensitivity.py:896-1051).

    Both passes run forwards in time and keep a running DFT (CWB_OP_DFT) at the nodes
    around `region` instead of a history: the forward run under the source, then per
    frequency an adjoint run under a decaying pulse with the same spectral load. The
    settled spectra of the two, paired as the triplet (z^-2, z^-1, 1) and the adjoint,
    drive the gradient kernel (CWB_OP_GRADIENT) once for the real and once for the
    imaginary half of the bilinear form. Exact once both runs have decayed;
    info["decay"] says how far they have, info["fit"] how spectral the cost is.
    """
    require_interior(sim, sensors, "sensor")
    require_interior(sim, source.position, "source")
    require_full_domain(sim)
    dev = device()
    frequencies = np.atleast_1d(np.asarray(frequencies, dtype=np.float64))
    logical = torch.zeros(sim.Nx_padded, dtype=torch.bool, device=dev)
    logical[tuple(slice(0, n) for n in sim.Nx)] = True
    region = logical if region is None else as_device(region, torch.bool)
    # the gradient at a node reads its neighbours, ghosts included, so the DFT does too
    kept = _dilated(sim, region, sim.reach + 1) & logical
    nodes = torch.stack(torch.nonzero(kept, as_tuple=True)).to(torch.int32)
    lin = flatten_indices(sim, nodes)
    num = lin.numel()

    mat = sim.build_materials(indicator)
    shot = prepare_shot(sim, mat, source.position, source.signal)
    require_off_held_walls(sim, shot.position)
    plan = sim.plan()
    N = sim.N
    material = sim.material(mat)
    grads = sim.gradient_fields(mat)
    grad_factors = [float(sim.np_dtype(float(f) / sim.dt**2)) for f in sim.step_factors()]

    host_table = phase_table(sim, frequencies)
    period = math.ceil(1.0 / (float(frequencies.min()) * sim.dt))
    # the same factors again over the last period alone, for how far the run settled
    tail = host_table.copy()
    tail[: N - period] = 0.0
    table = torch.as_tensor(np.concatenate((host_table, tail), axis=1), device=dev)
    table = table.to(sim.dtype).contiguous()
    F = len(frequencies)
    u_hat = torch.zeros((4 * F, num), dtype=sim.dtype, device=dev)
    U = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    sensor_lin = flatten_indices(sim, sensors)
    um = torch.zeros((N, sensor_lin.numel()), dtype=sim.dtype, device=dev)

    # ---------------------------------------------------------------- forward pass
    memory = pml_memory(sim, 3, dev)
    c = nat.level(U, add=0, period=2)
    ops = forward_ops(sim, mat, c, nat.level(U, add=1, period=2), c, shot, memory,
                      records=[(sensor_lin, um, 1, 0, nat.STORE_NATIVE)])
    ops.append(nat.op(nat.OP_DFT, a=c, points=nat.points(lin, table), g_mass=u_hat,
                      columns=4 * F))
    plan.march(ops, 0, N)
    del memory
    u_last = U[(N - 1) % 2].reshape(-1)[lin.long()].double().cpu().numpy()
    u_acc = u_hat.cpu().numpy()
    cost, dphi = _objective(objective, um)

    # ----------------------------------------------------------- adjoint excitation
    load, fit = spectral_load(sim, dphi, host_table)
    if fit > FIT_LIMIT[sim.precision]:
        raise ValueError(
            f"dcost/dtraces is off the sinusoids at {frequencies} by {fit:.1e}: the cost "
            f"is not spectral there, use sensitivity"
        )
    weights = sim.adjoint_weights(as_position(sim, sensors)).cpu().numpy().astype(np.float64)
    weight = sim.excitation_weights(mat, sensor_lin)

    # --------------------------------------------------------------- backward pass
    lam_hat = torch.zeros((4, num), dtype=sim.dtype, device=dev)
    fields = torch.zeros((4, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    flat_fields = fields.reshape(4, -1)
    gradient = nat.op(nat.OP_GRADIENT, a=nat.level(fields, mul=0, add=0),
                      b=nat.level(fields, mul=0, add=1), c=nat.level(fields, mul=0, add=2),
                      d=nat.level(fields, mul=0, add=3), mat=material, g_mass=grads["mass"],
                      g_stiff=grads["stiff"], scale=sim.adjoint_mass_factor(),
                      factors=grad_factors)
    decay = 0.0
    for f, frequency in enumerate(frequencies):
        signal = spectral_pulse(sim, frequency, load[f]) / weights
        signal = torch.as_tensor(signal, device=dev).to(sim.dtype).contiguous()
        U.zero_()
        lam_hat.zero_()
        # a fresh pml memory per run, from rest
        eta = pml_memory(sim, 5, dev)
        columns = [2 * f, 2 * f + 1, 2 * F + 2 * f, 2 * F + 2 * f + 1]
        ftable = table[:, columns].contiguous()
        ops = _adjoint_ops(sim, mat, U, eta, load=(sensor_lin, signal, weight))
        l0 = nat.level(U, add=0, period=2)
        ops.append(nat.op(nat.OP_REFILL, a=l0))
        ops.append(nat.op(nat.OP_DFT, a=l0, points=nat.points(lin, ftable), g_mass=lam_hat,
                          columns=4))
        plan.march(ops, 0, N)
        lam_last = U[(N - 1) % 2].reshape(-1)[lin.long()].double().cpu().numpy()

        spectrum, share = spectra(sim, u_acc[columns], u_last, frequency, period)
        adjoint_hat, adjoint_share = spectra(sim, lam_hat.cpu().numpy(), lam_last, frequency,
                                             period)
        decay = max(decay, share, adjoint_share)
        # lambda^t pairs with (u^(t - 2), u^(t - 1), u^t): the triplet is z^-2, z^-1, 1
        shift = np.exp(-2j * np.pi * frequency * sim.dt)
        triplet = (spectrum * shift**2, spectrum * shift, spectrum)
        # Re(a b) = Re a Re b - Im a Im b, the two halves of the bilinear form
        for part, sign in ((np.real, 1.0), (np.imag, -1.0)):
            values = np.stack([part(v) for v in (*triplet, sign * adjoint_hat)])
            flat_fields[:, lin.long()] = torch.as_tensor(values.astype(sim.np_dtype), device=dev)
            plan.march([gradient], 0, 1, graph=False)

    grads = frozen(sim, sim.finalize_gradients(grads))
    outside = ~region
    for g in grads.values():
        g[outside] = 0.0
    if decay > DECAY_LIMIT:
        warnings.warn(
            f"the last period still adds more than {DECAY_LIMIT:.0e} of the spectrum: the "
            f"gradient misses the tail the run cut off (info['decay'] says how much). "
            f"Lengthen the run or damp the faces.",
            RuntimeWarning,
            stacklevel=2,
        )
    return cost, grads, um, {"decay": decay, "fit": fit}


# ------------------------------------------------------------------- reconstruction
def reversible_damping(sim: Simulation, indicator, span: int) -> np.ndarray:
    """Damped nodes a reverse march of `span` steps can run backwards (cuwave sensitivity.py:139-157)."""
    from scipy import ndimage

    if sim.damping is None:
        return np.zeros(sim.Nx_padded, dtype=bool)
    minv = sim.inverse_inertia(indicator).cpu().numpy()
    minv = ndimage.maximum_filter(minv, size=3)
    damping = np.asarray(as_device(sim.damping, sim.dtype).cpu().numpy())
    dt = sim.np_dtype
    beta = dt(0.5) * dt(sim.dt) * damping * minv
    tiny = np.finfo(sim.np_dtype).tiny
    growth = dt(span) * np.log((dt(1.0) + beta) / np.maximum(dt(1.0) - beta, tiny))
    bound = math.log(REVERSIBLE_GROWTH[sim.precision])
    return (damping > 0) & (beta < 1.0) & (growth <= bound)


def reconstruction_nodes(sim: Simulation, indicator, span: int | None = None):
    """(strip, valid): the nodes a reverse march replays, and where it is exact (cuwave sensitivity.py:160-195).

    Irreversible are the pml nodes and the damped nodes too lossy to run backwards; the
    strip is the irreversible interior within `reach` (a Chebyshev dilation) of the
    reversible set, in C order.
    """
    from scipy import ndimage

    interior = np.zeros(sim.Nx_padded, dtype=bool)
    interior[tuple(slice(1, n - 1) for n in sim.Nx)] = True
    dev = device()
    if sim.damping is None and sim.pml is None:
        return torch.zeros((sim.ndim, 0), dtype=torch.int32, device=dev), torch.as_tensor(interior, device=dev)
    reversible = interior & ~pml_nodes(sim)
    if sim.damping is not None:
        span = sim.N if span is None else span
        damping = as_device(sim.damping, sim.dtype).cpu().numpy()
        reversible &= ~(damping > 0) | reversible_damping(sim, indicator, span)
    square = ndimage.generate_binary_structure(sim.ndim, sim.ndim)
    reach = ndimage.binary_dilation(reversible, structure=square, iterations=sim.reach, brute_force=True)
    strip = np.stack(np.nonzero(interior & ~reversible & reach)).astype(np.int32)
    return torch.as_tensor(strip, device=dev), torch.as_tensor(reversible, device=dev)


def segment_split(lo: int, hi: int, free: int) -> int:
    """The segment treeverse snapshots next when it must reverse segments lo .. hi - 1
    with `free` snapshot slots: binomial checkpointing (Griewank & Walther 2000,
    https://doi.org/10.1145/347837.347846; cuwave sensitivity.py:229-240). With s slots
    and r replays at most C(s + r, s) segments can be reversed; with the fewest replays
    r that cover hi - lo segments, the part past the snapshot is what s - 1 slots and r
    replays cover, C(s - 1 + r, s - 1) segments, so the snapshot sits that far before hi
    (and at least one segment past lo)."""
    need = hi - lo
    replays = next(r for r in itertools.count() if math.comb(free + r, free) >= need)
    return max(lo + 1, hi - math.comb(free - 1 + replays, free - 1))


def checkpoint_schedule(segments: int, slots: int) -> list[tuple]:
    """The treeverse schedule that reverses `segments` with `slots` snapshots beyond the
    initial state (the action sequence of cuwave sensitivity.py:243-269).

    Actions, in order: ("restore", k) and ("store", k) move segment k's start state
    between a snapshot and the working slots, ("drop", k) frees it, ("advance", a, b)
    marches from segment a's start to segment b's, and ("leaf", k) replays segment k
    forwards and then reverses it.

    Built with an explicit work stack. Reversing lo .. hi - 1 with free slots is: one
    segment, a leaf; no free slot, every segment from the last down re-marched from lo;
    otherwise march to the split, snapshot it, reverse the part past it with a slot
    fewer, drop the snapshot and reverse the part before it with the same slots.
    """
    actions: list[tuple] = []
    work: list[tuple] = [("reverse", 0, segments, slots)]
    while work:
        item = work.pop()
        if item[0] != "reverse":
            actions.append(item)
            continue
        _, lo, hi, free = item
        if hi - lo > 1 and free > 0:
            mid = segment_split(lo, hi, free)
            actions += [("restore", lo), ("advance", lo, mid), ("store", mid)]
            # popped last-in first: the part past the snapshot, its drop, the part before
            work += [("reverse", lo, mid, free), ("drop", mid), ("reverse", mid, hi, free - 1)]
            continue
        for k in range(hi - 1, lo, -1):
            actions += [("restore", lo), ("advance", lo, k), ("leaf", k)]
        actions += [("restore", lo), ("leaf", lo)]
    return actions


def _store_code(sim: Simulation, stored) -> int:
    if stored == sim.dtype:
        return nat.STORE_NATIVE
    return nat.STORE_BF16 if stored == BFLOAT16 else nat.STORE_F32


def reconstruction_sensitivity(sim: Simulation, source: Source, indicator, sensors,
                               objective: Callable, strip_dtype: str | None = None,
                               checkpoints: int | None = None, *, _mat: dict | None = None,
                               _probe: bool = False):
    """Cost and gradients as `sensitivity`, marching the forward field backwards behind a
    recorded strip instead of storing it (cuwave sensitivity.py:500-750).

    The lossless recursion run with its outer slots swapped steps the field backwards
    (a reversible damping negated); the nodes it cannot reverse (the pml layer, strong
    damping) are recorded each step over the strip that shields the rest, and replayed
    on the way back. With `checkpoints` the run is cut into segments replayed from
    snapshots on the treeverse schedule, so memory no longer grows with N.

    Returns (cost, grads, traces, info) with info = {"strip", "drift", "segment", "sweeps"}
    (and, with `_probe`, "source": d(cost)/d(source.signal) from the same adjoint march;
    `_mat` replaces the materials built from `indicator`).
    """
    require_interior(sim, sensors, "sensor")
    require_interior(sim, source.position, "source")
    require_full_domain(sim)
    if checkpoints is not None and checkpoints < 0:
        raise ValueError(f"checkpoints must be non-negative: {checkpoints}")
    stored = STRIP_DTYPES.get((strip_dtype, sim.precision), sim.dtype)
    if strip_dtype is not None and stored == sim.dtype:
        raise ValueError(
            f"strip_dtype {strip_dtype!r} is not narrower than {sim.precision}: "
            f"use 'bfloat16', or 'float32' under float64"
        )
    dev = device()
    N = sim.N
    mat = sim.build_materials(indicator) if _mat is None else _mat
    shot = prepare_shot(sim, mat, source.position, source.signal)
    require_off_held_walls(sim, shot.position)
    plan = sim.plan()
    lam = torch.zeros((N, shot.lin.numel()), dtype=sim.dtype, device=dev) if _probe else None
    itemsize = torch.empty(0, dtype=sim.dtype).element_size()
    stored_size = torch.empty(0, dtype=stored).element_size()

    U = torch.zeros((3, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    memory = pml_memory(sim, 3, dev)
    memory_list = [m for m in memory if m is not None]
    snapshot_bytes = 2 * U[0].numel() * itemsize + sum(m.numel() * itemsize for m in memory_list)
    strip, valid = reconstruction_nodes(sim, indicator)
    segment = N
    if checkpoints is not None and strip.shape[1]:
        row_bytes = 2 * strip.shape[1] * stored_size
        segment = min(N, max(2, snapshot_bytes // row_bytes))
    if segment < N:
        strip, valid = reconstruction_nodes(sim, indicator, segment)
    if not bool(valid.any()):
        raise ValueError(
            "damping too strong to reverse covers every interior node, so there is nothing "
            "to reconstruct; set checkpoints, damp only the faces with sponge, or use sensitivity"
        )
    num_strip = int(strip.shape[1])
    starts = list(range(0, N, segment)) + [N]
    lin_strip = flatten_indices(sim, strip) if num_strip else None
    store = _store_code(sim, stored)

    # backwards the layer sits behind the strip, and a reversible damping is negated
    back = replace(sim, pml=None)
    back_mat = dict(mat)
    if sim.damping is not None:
        back_mat["damping"] = torch.where(valid, -mat["damping"], mat["damping"]).contiguous()
    back_mat["profiles"] = [None, None, None]
    back_weight = back.excitation_weights(back_mat, shot.lin)
    back_shot = replace(shot, weight=back_weight)

    sensor_lin = flatten_indices(sim, sensors)
    sensor_weight = sim.excitation_weights(mat, sensor_lin)
    um = torch.zeros((N, sensor_lin.numel()), dtype=sim.dtype, device=dev)
    P = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    eta = pml_memory(sim, 5, dev)
    grads = sim.gradient_fields(mat)
    snapshots = {}
    state = {"recorded": 0, "steps": 0}
    grad_factors = [float(sim.np_dtype(float(f) / sim.dt**2)) for f in sim.step_factors()]

    def slot(i, mul=1, add=0):
        return nat.level(U, mul=mul, add=add, period=3)

    # ------------------------------------------------------------ forward pass
    def advance(a, b, buffer=None):
        records = []
        if a == state["recorded"]:
            records.append((sensor_lin, um, 1, 0, nat.STORE_NATIVE))
            state["recorded"] = b
        if buffer is not None:
            # buffer row r holds u^(seg_start - 2 + r); step t writes row t - seg_start + 2
            records.append((lin_strip, buffer[0], 1, buffer[1], store))
        ops = forward_ops(sim, mat, slot(0, add=0), slot(0, add=1), slot(0, add=2), shot,
                          memory, records=records)
        state["steps"] += b - a
        plan.march(ops, a, b - a)

    def slots_at(t):
        return U[t % 3], U[(t + 1) % 3]

    def store_snapshot(k):
        snapshots[k] = [f.clone() for f in (*slots_at(starts[k]), *memory_list)]

    def restore(k):
        for f, saved in zip((*slots_at(starts[k]), *memory_list), snapshots.get(k, ())):
            f.copy_(saved)
        if k == 0:
            for f in (*slots_at(0), *memory_list):
                f.zero_()

    # ----------------------------------------------------------- backward pass
    # triplet(m) = (u^(n-2), u^(n-1), u^n), n = N - 1 - m, sit in U[(N + 2 - m) % 3],
    # U[(N - m) % 3], U[(N + 1 - m) % 3]
    material = sim.material(mat)
    back_material = back.material(back_mat)

    def adjoint_ops(offset):
        """Adjoint step m + offset: lambda in P[(m + offset) % 2]."""
        l0 = nat.level(P, add=offset, period=2)
        l1 = nat.level(P, add=offset + 1, period=2)
        ops = []
        flags = 0
        if sim.pml is not None:
            ops.append(nat.op(nat.OP_PML_AUX, a=l1, mat=material, memory=eta))
            flags = nat.PML
        ops.append(nat.op(nat.OP_ADJOINT, flags=flags, a=l0, b=l1, mat=material, memory=eta,
                          scale=sim.adjoint_mass_factor()))
        ops.append(nat.op(nat.OP_EXCITE, a=l0,
                          points=nat.points(sensor_lin, state["signal"], weight=sensor_weight,
                                            row_add=offset)))
        if lam is not None:
            ops.append(nat.op(nat.OP_RECORD, a=l0, points=nat.points(shot.lin, lam, row_add=offset)))
        # the triplet of step m + offset and the lambda just stepped
        o_ = offset
        ops.append(nat.op(nat.OP_GRADIENT, a=slot(0, mul=-1, add=N + 2 - o_),
                          b=slot(0, mul=-1, add=N - o_), c=slot(0, mul=-1, add=N + 1 - o_),
                          d=l0, mat=material, g_mass=grads["mass"], g_stiff=grads["stiff"],
                          scale=sim.adjoint_mass_factor(), factors=grad_factors))
        return ops

    def leaf(k):
        s, e = starts[k], starts[k + 1]
        buffer = None
        if num_strip:
            buf = torch.zeros((e - s + 2, num_strip), dtype=stored, device=dev)
            if s:
                for row, f in enumerate(slots_at(s)):
                    buf[row] = narrow(f.reshape(-1)[lin_strip.long()], stored)
            buffer = (buf, 2 - s)
        advance(s, e, buffer)
        if "signal" not in state:
            state["cost"], dphi = _objective(objective, um)
            state["signal"] = adjoint_signal(sim, dphi, sensors)
        m0, m1 = N - e, N - s
        if not s:
            state["seed"] = float(torch.linalg.vector_norm(U[(N + 1 - m0) % 3] * valid))
        plan.march(adjoint_ops(0), m0, 1)
        if e - s > 1:
            # reverse step m beside adjoint step m + 1 (sequential here: they meet only
            # in the gradient)
            replay = None
            if num_strip:
                # u^(n-3), n = N - 1 - m, sits in row N - 2 - m - s of the buffer
                replay = nat.points(lin_strip, buf, row_mul=-1, row_add=N - 2 - s, store=store)
            ops = forward_ops(back, back_mat, slot(0, mul=-1, add=N), slot(0, mul=-1, add=N + 2),
                              slot(0, mul=-1, add=N + 1), back_shot, [None, None, None],
                              replay=replay, source_row=(-1, N - 2), fold=False)
            ops[0].mat = back_material
            ops += adjoint_ops(1)
            plan.march(ops, m0, e - s - 1)

    for action, *segs in checkpoint_schedule(len(starts) - 1, checkpoints or 0):
        if action == "advance":
            advance(starts[segs[0]], starts[segs[1]])
        elif action == "store":
            store_snapshot(segs[0])
        elif action == "restore":
            restore(segs[0])
        elif action == "drop":
            del snapshots[segs[0]]
        else:
            leaf(segs[0])

    grads = sim.finalize_gradients(grads)
    outside = ~valid
    for f in grads.values():
        f[outside] = 0.0
    seed = state["seed"]
    drift = float(torch.linalg.vector_norm(U[0] * valid)) / seed if seed > 0.0 else float("inf")
    info = {"strip": num_strip, "drift": drift, "segment": segment, "sweeps": state["steps"] / N}
    if lam is not None:
        info["source"] = (lam.flip(0) * sim.adjoint_weights(shot.position)).contiguous()
    return state["cost"], grads, um, info
