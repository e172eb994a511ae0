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
    """A grey design snapped to two phases: `low` where it lies below `eta`, `high`
    everywhere else (a NaN included), as cuwave's utils.threshold (utils.py:81-96).

    The result keeps the field's floating dtype (a float32 design stays float32, the
    precision the kernels read it in); a non-float field takes the dtype of the two
    phase values. numpy arrays and torch tensors come back as what they were.
    """
    if isinstance(field, torch.Tensor):
        kind = dtype or (field.dtype if field.is_floating_point() else torch.float64)
        snapped = torch.full(field.shape, high, dtype=kind, device=field.device)
        snapped[field < eta] = low
        return snapped
    values = np.asarray(field)
    kind = dtype or (values.dtype if values.dtype.kind == "f" else np.result_type(low, high))
    snapped = np.full(values.shape, high, dtype=kind)
    snapped[values < eta] = low
    return snapped


def resample(signal, dt: float, dt_new: float, N_new: int | None = None):
    """Linear interpolation of a sampled signal (time along axis 0) from step `dt` onto
    step `dt_new`, zero past its last sample (cuwave utils.py:99-134).

    Output row k sits at input position k * (dt_new / dt), the ratio and the positions
    in the signal's floating precision (float64 for an integer signal); it blends the
    two input rows around that position. Without `N_new` the output spans the input.
    numpy arrays and torch tensors come back as what they were.
    """
    given_torch = isinstance(signal, torch.Tensor)
    x = signal if given_torch else torch.from_numpy(np.ascontiguousarray(signal))
    count = x.shape[0]
    if count < 2:
        raise ValueError(f"resampling needs at least two samples, got {count}")
    if N_new is None:
        span = (count - 1) * dt / dt_new
        N_new = int(span + 1e-9 * max(1.0, span)) + 1
    real = x.dtype if x.is_floating_point() else torch.float64
    ratio = torch.tensor(dt_new / dt, dtype=real)
    position = torch.arange(N_new, dtype=real, device=x.device) * ratio.to(x.device)
    base = torch.floor(position).clamp(0, count - 2)
    frac = (position - base).reshape(N_new, *(1,) * (x.dim() - 1))
    i = base.to(torch.int64)
    x = x.to(real) if given_torch else x
    blended = (1 - frac) * x[i] + frac * x[i + 1]
    inside = (position <= count - 1).reshape(frac.shape)
    out = blended * inside
    return out if given_torch else out.numpy()


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
            devices: Sequence[int] | None = None, lanes: int | None = None) -> list[torch.Tensor]:
    """Receiver traces of every shot (cuwave utils.py:369-393), the shots side by side on
    `lanes` (see `misfit_gradient`)."""
    _one_device(devices)
    sources = list(sources)
    lanes = _lanes(sim, len(sources), simulate) if lanes is None else lanes
    return _on_lanes(sim, len(sources), lanes, lambda s, i: sensors.traces(
        simulate(s, sources[i], indicator, sensors=sensors.nodes)[1]))


def misfit(sim: Simulation, sources: Sequence[Source], indicator, sensors: Sensors, observed,
           objective: Callable = l2_misfit, devices: Sequence[int] | None = None,
           lanes: int | None = None) -> float:
    """The summed cost of `misfit_gradient`, forward passes only (cuwave utils.py:396-407)."""
    traces = measure(sim, sources, indicator, sensors, devices, lanes)
    return sum(objective(data)(t)[0] for t, data in zip(traces, observed))


def _on_lanes(sim: Simulation, count: int, lanes: int, work: Callable) -> list:
    """[work(sim, i) for i in range(count)], the items side by side on `lanes` lanes: a
    CUDA stream, a copy of `sim` (so a plan: step counter, graphs) and a host thread
    each, lane k taking items k, k + lanes, ...; the results in item order, their tensors
    usable on the caller's stream. The items must be independent."""
    lanes = max(1, min(int(lanes), count))
    if lanes <= 1:
        return [work(sim, i) for i in range(count)]
    from concurrent.futures import ThreadPoolExecutor
    from dataclasses import replace

    main = torch.cuda.current_stream()
    ready = torch.cuda.Event()
    ready.record(main)
    sims = [replace(sim) for _ in range(lanes)]
    streams = [torch.cuda.Stream(device=device()) for _ in range(lanes)]
    results: list = [None] * count

    def lane(k: int) -> torch.cuda.Event:
        stream = streams[k]
        stream.wait_event(ready)
        with torch.cuda.stream(stream):
            for i in range(k, count, lanes):
                results[i] = work(sims[k], i)
            done = torch.cuda.Event()
            done.record(stream)
        return done

    with ThreadPoolExecutor(max_workers=lanes) as pool:
        finished = list(pool.map(lane, range(lanes)))
    for done in finished:
        main.wait_event(done)

    def hand_over(x):
        if isinstance(x, torch.Tensor):
            x.record_stream(main)
        elif isinstance(x, (tuple, list)):
            for y in x:
                hand_over(y)

    for r in results:
        hand_over(r)
    return results


def _lanes(sim: Simulation, shots: int, solver: Callable) -> int:
    """Shots to run side by side: up to eight, as many as half the free device memory
    holds the fields of (`sensitivity` keeps N + 2 fields a shot)."""
    if shots <= 1:
        return 1
    field = int(np.prod(sim.Nx_padded)) * torch.empty((), dtype=sim.dtype).element_size()
    per_shot = (sim.N + 8) * field if solver is sensitivity else 16 * field
    free, _ = torch.cuda.mem_get_info(device())
    return int(max(1, min(8, shots, (free // 2) // max(per_shot, 1))))


def misfit_gradient(sim: Simulation, sources: Sequence[Source], indicator, sensors: Sensors,
                    observed, objective: Callable = l2_misfit,
                    adjoint: Callable = sensitivity, devices: Sequence[int] | None = None,
                    lanes: int | None = None):
    """Cost summed over the shots and its derivative with respect to `indicator` (cuwave utils.py:410-459).

    Each shot is one `adjoint` solve (`sensitivity`, or `reconstruction_sensitivity`
    where the history does not fit) with the receivers' objective lifted onto their
    corner nodes; the gradients are reparametrized onto the indicator and summed over
    the padded grid in shot order.

    The shots are independent, so `lanes` of them run side by side, each lane a CUDA
    stream with a plan of its own driven from its own host thread (by default as many
    as the free memory holds, at most eight); every shot's gradient is kept apart and the
    sum taken in shot order afterwards, so the result is the one-at-a-time result to the
    bit. `lanes=1` runs them in turn.
    """
    _one_device(devices)
    pairs = list(zip(sources, observed))
    lanes = _lanes(sim, len(pairs), adjoint) if lanes is None else max(1, min(int(lanes), len(pairs)))
    gradient = torch.zeros(sim.Nx_padded, dtype=sim.dtype, device=device())
    if lanes <= 1:
        cost = 0.0
        for source, data in pairs:
            shot_cost, grads, _, _ = adjoint(
                sim, source, indicator, sensors.nodes, sensors.objective(objective(data))
            )
            cost += shot_cost
            gradient += _reparametrize(sim, indicator, grads)
        return cost, gradient

    def shot(s: Simulation, i: int):
        source, data = pairs[i]
        shot_cost, grads, _, _ = adjoint(s, source, indicator, sensors.nodes,
                                         sensors.objective(objective(data)))
        return shot_cost, _reparametrize(sim, indicator, grads)

    cost = 0.0
    for shot_cost, shot_gradient in _on_lanes(sim, len(pairs), lanes, shot):
        cost += shot_cost
        gradient += shot_gradient
    return cost, gradient


# ------------------------------------------------------------------------------ tato
def energy(sim: Simulation) -> Callable:
    """The objective that scores the energy reaching the sensors (cuwave utils.py:463-470):
    J = (dx^ndim dt / 2) sum over steps and sensors of p^2, dJ/dp = dx^ndim dt p."""
    cell_time = float(np.prod(sim.dx)) * sim.dt

    def objective(traces):
        gradient = cell_time * traces
        return 0.5 * cell_time * float(torch.sum(traces**2)), gradient

    return objective


def response(sim: Simulation, source: Source, indicator, sensors, objective: Callable):
    """One shot forward only: its cost and its final field over the logical grid
    (cuwave utils.py:473-487)."""
    field, traces = simulate(sim, source, indicator, sensors=sensors)
    cost, _ = objective(traces)
    return cost, field


def response_gradient(sim: Simulation, source: Source, indicator, sensors, objective: Callable,
                      adjoint: Callable = sensitivity):
    """One shot's cost and its gradient on the design field, taken by `adjoint`
    (`sensitivity`, or `reconstruction_sensitivity` where a stored history does not fit)
    and mapped from (mass, stiffness) onto the design (cuwave utils.py:490-514)."""
    cost, grads, _, _ = adjoint(sim, source, indicator, sensors, objective)
    return cost, _reparametrize(sim, indicator, grads)


# ------------------------------------------------------------------------------ tpto
def intensity(sim: Simulation, frequencies, weights=None) -> Callable:
    """The objective that scores spectral intensity at the sensors (cuwave utils.py:518-552):
    J = sum over frequencies and sensors of w |u(f)|^2, u(f) = dt sum_t u(t) exp(-2 pi i f t dt).

    The transform is one real matrix, its rows the cosine and the negated sine rows of
    every frequency (phases in float64, since they reach 1e5 radians over a long run,
    then rounded to the simulation's precision), so J's derivative is that matrix
    transposed onto 2 w (Re, Im).
    """
    f = np.atleast_1d(np.asarray(frequencies, dtype=np.float64))
    phase = 2.0 * np.pi * np.outer(f, np.arange(sim.N, dtype=np.float64) * sim.dt)
    dev = device()
    table = torch.as_tensor(np.concatenate([np.cos(phase), -np.sin(phase)]), device=dev).to(sim.dtype)
    dt = float(sim.np_dtype(sim.dt))
    count = f.size
    w = torch.ones((), dtype=sim.dtype, device=dev) if weights is None else as_device(weights, sim.dtype)

    def objective(traces):
        spectrum = dt * (table @ traces)  # (2F, sensors): the Re rows over the Im rows
        re, im = spectrum[:count], spectrum[count:]
        cost = float(torch.sum(w * (re * re + im * im)))
        both = torch.broadcast_to(w, re.shape).repeat(2, 1)
        return cost, 2.0 * dt * (table.T @ (both * spectrum))

    return objective


# ------------------------------------------------------------------- time dispersion
def _warn_low_order(sim: Simulation) -> None:
    """At space order 2 the leapfrog time error cancels part of the spatial one, so
    taking it out makes the solution worse: say so."""
    if sim.space_order == 2:
        warnings.warn(
            "removing the leapfrog time error at space_order 2 makes the result less "
            "accurate (there it offsets the spatial error); use space_order 4 or higher",
            RuntimeWarning,
            stacklevel=3,
        )


def _warp(sim: Simulation, values, offset: int, read: Callable):
    """`values` (time along axis 0, row n at time (n + offset) dt) with its spectrum moved
    from each frequency w onto read(w) (NaN: no counterpart, dropped), back on the same
    rows (cuwave utils.py:567-590).

    The moved spectrum is a non-uniform transform from the sample times onto read(w) over
    the bins of a real FFT twice the signal's length (so a moved sample cannot wrap round
    into the kept rows), evaluated as phase matrices in float64 a bounded number of
    entries at a time, then inverted by that FFT.
    """
    given_torch = isinstance(values, torch.Tensor)
    x = values if given_torch else torch.from_numpy(np.ascontiguousarray(values))
    count = x.shape[0]
    flat = x.reshape(count, -1)
    length = 2 * count
    omega = 2.0 * np.pi * np.fft.rfftfreq(length, sim.dt)
    moved = read(omega)
    valid = np.isfinite(moved)
    ctype = torch.complex64 if flat.dtype == torch.float32 else torch.complex128
    dev = flat.device
    times = torch.as_tensor((offset + np.arange(count)) * sim.dt, device=dev)
    targets = torch.as_tensor(np.where(valid, moved, 0.0), device=dev)
    samples = flat.to(ctype)
    rows_per_chunk = max(1, (1 << 23) // count)  # phase entries held at once
    spectrum = torch.cat([
        torch.exp(-1j * torch.outer(targets[k:k + rows_per_chunk], times)).to(ctype) @ samples
        for k in range(0, omega.size, rows_per_chunk)
    ])
    back = torch.as_tensor(valid * np.exp(1j * omega * offset * sim.dt), device=dev).to(ctype)
    out = torch.fft.irfft(spectrum * back[:, None], length, dim=0)[:count].to(x.dtype).reshape(x.shape)
    return out if given_torch else out.numpy()


def tdt(sim: Simulation, signal, offset: int = 0):
    """The time-dispersion transform (cuwave utils.py:593-609): what leapfrog must be fed
    for `signal` to come out free of its time error, each frequency w read at the
    leapfrog's (2 / dt) sin(w dt / 2). offset 0 for a source signal, 1 for a record."""
    _warn_low_order(sim)
    return _warp(sim, signal, offset, lambda w: np.sin(0.5 * sim.dt * w) * (2.0 / sim.dt))


def itdt(sim: Simulation, record, offset: int = 1):
    """The inverse of `tdt` (cuwave utils.py:612-634): each frequency w read at
    (2 / dt) arcsin(w dt / 2), nothing where w dt / 2 passes 1 (above what leapfrog can
    carry at this dt). offset 1 for a record of `simulate`, 0 for a source signal."""
    _warn_low_order(sim)

    def read(w):
        s = 0.5 * sim.dt * w
        return np.where(s <= 1.0, np.arcsin(np.clip(s, None, 1.0)) * (2.0 / sim.dt), np.nan)

    return _warp(sim, record, offset, read)


def leapfrog_frequency(sim: Simulation, frequency) -> np.ndarray:
    """The frequency whose leapfrog solution oscillates at `frequency` exactly
    (cuwave utils.py:637-643): arcsin(pi f dt) / (pi dt), defined below 1 / (pi dt)."""
    _warn_low_order(sim)
    x = np.pi * sim.dt * np.asarray(frequency, dtype=np.float64)
    if np.any(x >= 1.0):
        raise ValueError(f"{frequency} is above 1 / (pi dt) = {1 / (np.pi * sim.dt):g}")
    return np.arcsin(x) / (np.pi * sim.dt)
