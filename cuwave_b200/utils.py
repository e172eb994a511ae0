"""Shot glue around the hot path: off-node sources and receivers, and the multi-shot costs.

Restates the scalar part of cuwave `utils.py`: coordinates between grid nodes reach the
kernels as the 2**ndim corners of their cell with multilinear weights (`distribute`,
utils.py:144-247), a `Source` built from them (`point_source`, utils.py:250-277) and its
transpose (`collect_source`, utils.py:280-299), receivers at arbitrary coordinates
(`Sensors`, utils.py:326-365), and the inversion drivers that sum a cost and its
reparametrized gradient over a shot list (`measure`, `misfit`, `misfit_gradient`,
utils.py:369-459), with the objectives and small signal helpers beside them.

The weights are made on the host in float64 and cast once, as the reference does, and
the corner sums of `Sensors.traces` / `collect_source` add the corners in the order
numpy's float reduction takes over a row of 4 or 8 (`corner_sum`), so the receiver
traces and the gradients that follow from them match the reference's CPU run bit for
bit. Several receivers or shots may share a corner node; the step kernels add their
loads there atomically, so such shared nodes sum in an unspecified order, as on the
reference's GPU path.
"""

from __future__ import annotations

import itertools
import warnings
from collections.abc import Callable, Sequence

import numpy as np
import torch

from .sensitivity import l2_misfit, sensitivity
from .wave import Simulation, Source, as_device, device, simulate

TOL = 1e-6  # in index units: a coordinate this far past a wall still counts as on it


# --------------------------------------------------------------------------- helpers
def _reparametrize(sim: Simulation, indicator, grads: dict) -> torch.Tensor:
    """d(cost)/d(mass, stiff) chained onto the indicator (cuwave utils.py:19-24)."""
    d_mass, d_stiff = sim.parametrization_jacobian(indicator)
    return d_mass * grads["mass"] + d_stiff * grads["stiff"]


def _one_device(devices: Sequence[int] | None) -> None:
    """Accept a device list that names the current GPU only: its shots run in sequence.

    The reference spreads shots over several GPUs, a GPU listed twice running two at
    once (utils.py:50-73); a repeated entry changes only the schedule, not the result,
    and this build steps the scalar path on one GPU.
    """
    if devices is None:
        return
    here = device().index or 0
    others = sorted({int(d) for d in devices} - {here})
    if others:
        raise NotImplementedError(
            f"devices {tuple(devices)} name GPUs {others} besides the current one ({here}); "
            "the scalar path runs on one GPU"
        )


def corner_sum(values: torch.Tensor, pairwise: bool = True) -> torch.Tensor:
    """Sum over the last axis in the order numpy's float reduction takes.

    With the summed axis contiguous (`pairwise`), numpy adds a row of n < 8 elements
    one after another onto 0; from 8 to 128 it keeps eight running sums, adds them
    pairwise, then the remainder one after another. With the summed axis strided (a
    record gathered column-major) it adds the slices one after another. Restating both
    makes the corner sums agree with the reference's host arithmetic exactly.
    """
    n = values.shape[-1]
    if n < 8 or not pairwise:
        out = values[..., 0] + 0.0
        for k in range(1, n):
            out = out + values[..., k]
        return out
    if n > 128:
        raise ValueError(f"a corner row of {n} values: at most 128")
    r = [values[..., j] for j in range(8)]
    whole = n - n % 8
    for i in range(8, whole, 8):
        r = [r[j] + values[..., i + j] for j in range(8)]
    out = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]))
    out = out + 0.0
    for i in range(whole, n):
        out = out + values[..., i]
    return out


def _row_major(table: torch.Tensor) -> bool:
    """Whether numpy would sum the corners of this (N, columns) table along contiguous rows."""
    return table.shape[0] == 1 or table.stride(-1) == 1


# --------------------------------------------------------------------------- general
def interior_slice(sim: Simulation) -> tuple[slice, ...]:
    """The interior nodes, without the ghost ring or the padding (cuwave utils.py:76-78)."""
    return tuple(slice(1, n - 1) for n in sim.Nx)


def threshold(field, eta: float = 0.5, low: float = 0.0, high: float = 1.0, dtype=None):
    """`low` below `eta`, `high` from it on, in the field's float dtype (cuwave utils.py:81-96)."""
    if isinstance(field, torch.Tensor):
        if dtype is None:
            dtype = field.dtype if field.is_floating_point() else torch.float64
        return torch.where(field < eta, low, high).to(dtype)
    field = np.asarray(field)
    snapped = np.where(field < eta, low, high)
    if dtype is None:
        dtype = field.dtype if field.dtype.kind == "f" else snapped.dtype
    return snapped.astype(dtype)


def resample(signal, dt: float, dt_new: float, N_new: int | None = None):
    """Linear resampling from step `dt` to `dt_new`, zero past the end (cuwave utils.py:99-134).

    Works on numpy arrays and torch tensors alike, returning the kind it was given.
    """
    is_torch = isinstance(signal, torch.Tensor)
    values = signal if is_torch else np.asarray(signal)
    steps = values.shape[0]
    if steps < 2:
        raise ValueError(f"resampling needs at least two samples, got {steps}")
    if N_new is None:
        span = (steps - 1) * dt / dt_new
        N_new = int(span + 1e-9 * max(1.0, span)) + 1
    if is_torch:
        dtype = values.dtype if values.is_floating_point() else torch.float64
        ratio = torch.tensor(dt_new / dt, dtype=dtype).item()
        t = torch.arange(N_new, dtype=dtype, device=values.device) * ratio
        left = torch.clamp(torch.floor(t), 0, steps - 2)
        index = left.to(torch.int64)
        vals = values.to(dtype)
    else:
        dtype = np.dtype(values.dtype if values.dtype.kind == "f" else np.float64)
        t = np.arange(N_new, dtype=dtype) * dtype.type(dt_new / dt)
        left = np.clip(np.floor(t), 0, steps - 2)
        index = left.astype(np.int32)
        vals = values
    weight = t - left
    if values.ndim > 1:
        weight = weight.reshape(N_new, *(1,) * (values.ndim - 1))
    interpolated = (1 - weight) * vals[index] + weight * vals[index + 1]
    return interpolated * (t.reshape(weight.shape) <= steps - 1)


def line(start, stop, count: int) -> np.ndarray:
    """`count` coordinates from `start` to `stop`, both ends included (cuwave utils.py:137-141)."""
    return np.linspace(start, stop, count)


def _corner_weights(sim: Simulation, coords: np.ndarray, shift: np.ndarray):
    """Cell corners and multilinear weights of `coords` (cuwave utils.py:144-182).

    Returns (nodes, weights) shaped (ndim, num, 2**ndim) and (num, 2**ndim): the lowest
    corner clipped so that the cell's far corner is still interior, the corners in
    binary order with axis 0 slowest.
    """
    index = np.empty_like(coords)
    for d in range(sim.ndim):
        nodal = coords[:, d] / sim.dx[d] + 1.0
        if nodal.min() < 1.0 - TOL or nodal.max() > sim.Nx[d] - 2.0 + TOL:
            length = (sim.Nx[d] - 3) * sim.dx[d]
            raise ValueError(
                f"axis {d} coordinate outside the domain [0, {length:g}]: "
                f"[{float(coords[:, d].min()):g}, {float(coords[:, d].max()):g}]"
            )
        staggered = float(shift[d] > 0.0)
        index[:, d] = np.clip(nodal - shift[d], 1.0, sim.Nx[d] - 2.0 - staggered)
    base = np.stack([
        np.clip(np.floor(index[:, d]), 1, sim.Nx[d] - 3 - (shift[d] > 0.0)).astype(np.int32)
        for d in range(sim.ndim)
    ])
    offset = index.T - base
    corners = np.array(list(itertools.product((0, 1), repeat=sim.ndim)))
    nodes = base[:, :, None] + corners.T[:, None, :]
    weights = np.ones((len(coords), len(corners)))
    for d in range(sim.ndim):
        frac = offset[d][:, None]
        weights *= np.where(corners[None, :, d] == 1, frac, 1.0 - frac)
    return nodes, weights


def cell_corners(sim: Simulation, coords, direction=None):
    """Host half of `distribute`: int32 nodes (ndim, num * 2**ndim) and float64 weights (num, 2**ndim)."""
    coords = np.atleast_2d(np.asarray(coords, dtype=float))
    if coords.shape[1] != sim.ndim:
        raise ValueError(f"coordinates need {sim.ndim} components, not {coords.shape[1]}")
    ncomp = getattr(sim, "ncomp", 1)
    shifts = getattr(sim, "component_offsets", None)
    if shifts is None:
        shifts = np.zeros((ncomp, sim.ndim))
    if direction is None and ncomp > 1:
        raise ValueError(f"a {ncomp}-component unknown needs a direction")
    nodes, weights = _corner_weights(sim, coords, np.asarray(shifts[0], dtype=float))
    if direction is not None:
        n = np.atleast_2d(np.asarray(direction, dtype=float))
        if n.shape[1] != ncomp:
            raise ValueError(f"direction needs {ncomp} components, not {n.shape[1]}")
        if len(n) == 1:
            n = np.repeat(n, len(coords), axis=0)
        if len(n) != len(coords):
            raise ValueError(f"{len(n)} directions for {len(coords)} coordinates")
        weights = weights * n[:, :1]
    return nodes.reshape(sim.ndim, -1).astype(np.int32), weights


def distribute(sim: Simulation, coords, direction=None):
    """Multilinear interpolation of physical `coords` onto the grid (cuwave utils.py:185-247).

    Args:
        sim: the simulation whose grid the coordinates land on.
        coords: (num, ndim) physical coordinates, node 1 at the origin.
        direction: (1,) or (num, 1) factors on the weights; the scalar unknown has one
            component, so a direction is a scale.

    Returns:
        (nodes, weights): (ndim, num * 2**ndim) int32 grid indices and (num, 2**ndim)
        weights in the simulation's dtype, both on the GPU.
    """
    nodes, weights = cell_corners(sim, coords, direction)
    dev = device()
    return (
        torch.as_tensor(nodes, device=dev),
        torch.as_tensor(weights, device=dev).to(sim.dtype),
    )


def spread_columns(signal: torch.Tensor, weights: torch.Tensor, volume: float) -> torch.Tensor:
    """(N, num) signals times the (num, K) corner weights over the cell volume: (N, num * K).

    The product is taken in the weights' dtype and divided by the float64 volume before
    rounding back, as numpy does for the reference.
    """
    columns = (signal[:, :, None] * weights).reshape(signal.shape[0], -1)
    return (columns.to(torch.float64) / volume).to(weights.dtype).contiguous()


def gather_columns(columns: torch.Tensor, weights: torch.Tensor, volume: float) -> torch.Tensor:
    """Transpose of `spread_columns`: (N, num * K) -> (N, num), divided by the volume in the weights' dtype."""
    pairwise = _row_major(columns)
    columns = columns.reshape(columns.shape[0], weights.shape[0], -1)
    volume = torch.tensor(volume, dtype=weights.dtype).item()
    return corner_sum(columns * weights, pairwise) / volume


def point_source(sim: Simulation, coords, signal, direction=None) -> Source:
    """A `Source` firing `signal` at `coords`, spread over the cell corners (cuwave utils.py:250-277).

    `signal` is one (N,) trace for every coordinate or (N, num), one each; the columns
    are divided by the cell volume so the amplitude does not depend on the spacing.
    """
    nodes, weights = distribute(sim, coords, direction)
    count = weights.shape[0]
    signal = as_device(signal, sim.dtype)
    if signal.dim() == 1:
        signal = signal[:, None].expand(signal.shape[0], count)
    if signal.shape[1] != count:
        raise ValueError(f"{signal.shape[1]} signal columns for {count} sources")
    return Source(nodes, spread_columns(signal, weights, float(np.prod(sim.dx))))


def collect_source(sim: Simulation, coords, columns, direction=None) -> torch.Tensor:
    """Transpose of `point_source`: (N, num * 2**ndim) node columns onto the (N, num) signals (cuwave utils.py:280-299)."""
    _, weights = distribute(sim, coords, direction)
    return gather_columns(as_device(columns, sim.dtype), weights, float(np.prod(sim.dx)))


def shots(sim: Simulation, coords, signal, direction=None) -> list[Source]:
    """One single-coordinate `Source` per coordinate (cuwave utils.py:302-309)."""
    return [point_source(sim, c, signal, direction) for c in np.atleast_2d(coords)]


def stack(sources: Sequence[Source]) -> Source:
    """Several shots fired in one simulation: positions and columns side by side (cuwave utils.py:312-323).

    Encode the shots (random signs, phase shifts) by scaling their signals first.
    """
    dev = device()
    position = torch.cat([as_device(s.position, torch.int32) for s in sources], dim=1)
    signal = torch.cat([torch.as_tensor(s.signal).to(dev) for s in sources], dim=1)
    return Source(position, signal.contiguous())


class Sensors:
    """Receivers at arbitrary coordinates, read through their cell corners (cuwave utils.py:326-365).

    `nodes` (ndim, count * 2**ndim) go to `simulate` / `sensitivity` as the sensor
    positions; `traces` folds that node record onto the receivers and `scatter` is its
    transpose.
    """

    def __init__(self, sim: Simulation, coords, direction=None) -> None:
        self.sim = sim
        self.coordinates = np.atleast_2d(np.asarray(coords, dtype=float))
        self.count = len(self.coordinates)
        self.nodes, self.weights = distribute(sim, self.coordinates, direction)

    def traces(self, record: torch.Tensor) -> torch.Tensor:
        """(N, count * 2**ndim) node record -> (N, count) receiver traces."""
        values = record.reshape(record.shape[0], self.count, -1) * self.weights
        return corner_sum(values, _row_major(record))

    def scatter(self, dphi: torch.Tensor) -> torch.Tensor:
        """Transpose of `traces`: (N, count) -> (N, count * 2**ndim)."""
        dphi = as_device(dphi, self.weights.dtype)
        return (dphi[:, :, None] * self.weights).reshape(dphi.shape[0], -1)

    def objective(self, objective: Callable) -> Callable:
        """A receiver-space objective lifted onto the node record the adjoint reads."""

        def wrapped(record):
            cost, dphi = objective(self.traces(record))
            return cost, self.scatter(dphi)

        return wrapped


# ------------------------------------------------------------------------------- fwi
def measure(sim: Simulation, sources: Sequence[Source], indicator, sensors: Sensors,
            devices: Sequence[int] | None = None) -> list[torch.Tensor]:
    """Receiver traces of every shot (cuwave utils.py:369-393)."""
    _one_device(devices)
    return [
        sensors.traces(simulate(sim, source, indicator, sensors=sensors.nodes)[1])
        for source in sources
    ]


def misfit(sim: Simulation, sources: Sequence[Source], indicator, sensors: Sensors, observed,
           objective: Callable = l2_misfit, devices: Sequence[int] | None = None) -> float:
    """The summed cost of `misfit_gradient`, forward passes only (cuwave utils.py:396-407)."""
    traces = measure(sim, sources, indicator, sensors, devices)
    return sum(objective(data)(t)[0] for t, data in zip(traces, observed))


def misfit_gradient(sim: Simulation, sources: Sequence[Source], indicator, sensors: Sensors,
                    observed, objective: Callable = l2_misfit,
                    adjoint: Callable = sensitivity, devices: Sequence[int] | None = None):
    """Cost summed over the shots and its derivative with respect to `indicator` (cuwave utils.py:410-459).

    Each shot is one `adjoint` solve (`sensitivity`, or `reconstruction_sensitivity`
    where the history does not fit) with the receivers' objective lifted onto their
    corner nodes; the gradients are reparametrized onto the indicator and summed over
    the padded grid in shot order.
    """
    _one_device(devices)
    cost = 0.0
    gradient = torch.zeros(sim.Nx_padded, dtype=sim.dtype, device=device())
    for source, data in zip(sources, observed):
        shot_cost, grads, _, _ = adjoint(
            sim, source, indicator, sensors.nodes, sensors.objective(objective(data))
        )
        cost += shot_cost
        gradient += _reparametrize(sim, indicator, grads)
    return cost, gradient


# ------------------------------------------------------------------------------ tato
def energy(sim: Simulation) -> Callable:
    """Objective: J = 1/2 sum over sensors and steps of p^2, times dx^ndim dt (cuwave utils.py:463-470)."""
    scale = float(np.prod(sim.dx)) * sim.dt

    def objective(traces):
        return 0.5 * scale * float(torch.sum(traces**2)), scale * traces

    return objective


def response(sim: Simulation, source: Source, indicator, sensors, objective: Callable):
    """(cost, final field) of one forward pass (cuwave utils.py:473-487)."""
    wavefield, traces = simulate(sim, source, indicator, sensors=sensors)
    return objective(traces)[0], wavefield


def response_gradient(sim: Simulation, source: Source, indicator, sensors, objective: Callable,
                      adjoint: Callable = sensitivity):
    """Cost of one shot and its reparametrized gradient (cuwave utils.py:490-514)."""
    cost, grads, _, _ = adjoint(sim, source, indicator, sensors, objective)
    return cost, _reparametrize(sim, indicator, grads)


# ------------------------------------------------------------------------------ tpto
def intensity(sim: Simulation, frequencies, weights=None) -> Callable:
    """Objective: J = sum w |u_hat(f)|^2 over the sensors (cuwave utils.py:518-552).

    u_hat(f) = dt sum_t u(t) e^{-2 pi i f t dt}, with the phase tables built in float64
    and cast to the simulation's dtype; the derivative is the same tables read back.
    """
    f = np.atleast_1d(np.asarray(frequencies, dtype=np.float64))
    t = np.arange(sim.N, dtype=np.float64) * sim.dt
    phase = 2.0 * np.pi * t[:, None] * f[None, :]
    dev = device()
    cos = torch.as_tensor(np.cos(phase), device=dev).to(sim.dtype)
    sin = torch.as_tensor(np.sin(phase), device=dev).to(sim.dtype)
    scale = float(sim.np_dtype(sim.dt))
    w = 1.0 if weights is None else as_device(weights, sim.dtype)

    def objective(traces):
        re = scale * (cos.T @ traces)
        im = -scale * (sin.T @ traces)
        cost = float(torch.sum(w * (re * re + im * im)))
        return cost, 2.0 * scale * (cos @ (w * re) - sin @ (w * im))

    return objective


# ------------------------------------------------------------------- time dispersion
def _warn_low_order(sim: Simulation) -> None:
    if sim.space_order == 2:
        warnings.warn(
            "at space_order 2 the leapfrog time error offsets the spatial one, so removing "
            "it makes the result less accurate; use space_order 4 or higher",
            RuntimeWarning,
            stacklevel=3,
        )


def _warp(sim: Simulation, values, offset: int, read: Callable):
    """The spectrum of `values` re-read at `read(omega)`, back on the same rows (cuwave utils.py:567-590).

    A direct transform from the sample times onto the warped frequencies (tables in
    float64), then an inverse real FFT of twice the length, so the moved samples do not
    wrap round.
    """
    is_torch = isinstance(values, torch.Tensor)
    x = values if is_torch else torch.as_tensor(np.asarray(values))
    rows = x.reshape(x.shape[0], -1)
    steps = rows.shape[0]
    size = 2 * steps
    omega = 2.0 * np.pi * np.fft.rfftfreq(size, sim.dt)
    target = read(omega)
    keep = np.isfinite(target)
    cdtype = torch.complex64 if rows.dtype == torch.float32 else torch.complex128
    times = torch.as_tensor((np.arange(steps) + offset) * sim.dt, device=rows.device)
    freqs = torch.as_tensor(np.where(keep, target, 0.0), device=rows.device)
    crow = rows.to(cdtype)
    spectrum = torch.empty((omega.size, rows.shape[1]), dtype=cdtype, device=rows.device)
    block = max(1, 2**23 // steps)
    for k in range(0, omega.size, block):
        table = torch.exp(-1j * torch.outer(freqs[k:k + block], times))
        spectrum[k:k + block] = table.to(cdtype) @ crow
    shift = torch.as_tensor(keep * np.exp(1j * omega * offset * sim.dt), device=rows.device)
    out = torch.fft.irfft(spectrum * shift.to(cdtype)[:, None], size, dim=0)[:steps]
    out = out.to(x.dtype).reshape(x.shape)
    return out if is_torch else out.numpy()


def tdt(sim: Simulation, signal, offset: int = 0):
    """Time-dispersion transform: the input leapfrog needs for `signal` to come out exact (cuwave utils.py:593-609)."""
    _warn_low_order(sim)
    return _warp(sim, signal, offset, lambda w: 2.0 / sim.dt * np.sin(0.5 * w * sim.dt))


def itdt(sim: Simulation, record, offset: int = 1):
    """Inverse of `tdt`, zero above the highest frequency leapfrog carries (cuwave utils.py:612-634)."""
    _warn_low_order(sim)

    def read(omega):
        half = 0.5 * omega * sim.dt
        inverse = 2.0 / sim.dt * np.arcsin(np.minimum(half, 1.0))
        return np.where(half <= 1.0, inverse, np.nan)

    return _warp(sim, record, offset, read)


def leapfrog_frequency(sim: Simulation, frequency) -> np.ndarray:
    """The leapfrog frequency that answers exactly for `frequency` (cuwave utils.py:637-643)."""
    _warn_low_order(sim)
    phase = np.pi * np.asarray(frequency, dtype=np.float64) * sim.dt
    if np.any(phase >= 1.0):
        raise ValueError(f"{frequency} is above 1 / (pi dt) = {1 / (np.pi * sim.dt):g}")
    return np.arcsin(phase) / (np.pi * sim.dt)
