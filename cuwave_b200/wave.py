"""The grid, its configuration and the forward march: `Simulation`, `Source`, `simulate`.

Restates cuwave `wave.py` for the scalar path: the padded C-contiguous layout
(`padded_shape`, wave.py:120-122), the ghost conventions (`mirror_ghosts`,
wave.py:125-134), flat indices (`flatten_indices`, wave.py:364-382), the cell weights
(wave.py:336-354) and `simulate` (wave.py:1071-1163) with the same arguments and
return. Arrays are torch tensors on the current CUDA device; the time loop runs in the
native library (`cwb_march`), chunks of steps replayed as CUDA graphs.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np
import torch

from . import _native as nat
from .boundary import (
    Dirichlet,
    Neumann,
    Pml,
    canonical_boundary,
    face_mask,
    faces_with,
    pml_profiles,
    pml_widths,
    validate_pml,
)
from .stencils import STENCILS, operator_row, stable_dt  # noqa: F401  (re-export)

# a record of this dtype holds bfloat16: the high half of each float32
BFLOAT16 = torch.uint16
# cell codes of a masked domain (cuwave wave.py:662-663)
CELL_DEEP = 1 << 30  # a node whose cells all take the full radius
CELL_HELD = 7  # the radius code of a cell open onto a node held at zero


def padded_shape(Nx: tuple[int, ...]) -> tuple[int, ...]:
    """The fastest axis padded to a multiple of 32 (cuwave wave.py:120-122)."""
    return (*Nx[:-1], ((Nx[-1] + 31) // 32) * 32)


def device() -> torch.device:
    return nat.require_cuda()


def as_device(values, dtype: torch.dtype, *, copy: bool = False) -> torch.Tensor:
    """`values` (tensor, numpy array or sequence) as a contiguous tensor on the GPU."""
    dev = device()
    if isinstance(values, torch.Tensor):
        out = values.to(device=dev, dtype=dtype, non_blocking=True)
        if copy and out is values:
            out = out.clone()
        return out.contiguous()
    return torch.as_tensor(np.ascontiguousarray(values), dtype=dtype, device=dev)


@dataclass
class Source:
    """A shot: `position` (ndim, num_sources) grid indices, `signal` (N, num_sources)."""

    position: Any
    signal: Any


@dataclass
class Simulation:
    """Grid, timestepping and configuration of the scalar step (cuwave wave.py:479-630).

    `threads` is accepted for compatibility with the reference's signature; the native
    kernels choose their own launch shapes. `domain` (the nodes stepped) and `dirichlet`
    (the nodes held at zero) are boolean masks over the padded grid, graded at their
    walls (`domain_cells`); `devices` names one GPU at most.
    """

    Nx: tuple[int, ...]
    dx: tuple[float, ...]
    N: int
    dt: float
    threads: tuple[int, ...] | None = None
    precision: str = "float32"
    space_order: int = 2
    stencil: str = "optimized"
    boundary: tuple = None
    damping: Any = None
    domain: Any = None
    dirichlet: Any = None
    pml: Pml | None = None
    devices: tuple[int, ...] | None = None

    default_boundary = Neumann
    derive_inertia = False

    def __post_init__(self) -> None:
        self.Nx = tuple(int(n) for n in self.Nx)
        self.dx = tuple(float(d) for d in self.dx)
        self.ndim = len(self.Nx)
        self.Nx_padded = padded_shape(self.Nx)
        strides = [1] * self.ndim
        for d in range(self.ndim - 2, -1, -1):
            strides[d] = strides[d + 1] * self.Nx_padded[d + 1]
        self.strides = tuple(strides)
        if self.precision not in ("float32", "float64"):
            raise ValueError(f"precision is float32 or float64: {self.precision!r}")
        self.dtype = torch.float32 if self.precision == "float32" else torch.float64
        self.np_dtype = np.float32 if self.precision == "float32" else np.float64
        self.boundary = canonical_boundary(self.boundary, self.ndim, self.default_boundary)
        if self.space_order % 2 != 0 or self.space_order < 2:
            raise ValueError("space_order must be an even integer >= 2")
        if self.space_order > 16:
            raise NotImplementedError("the kernels step radius 1 .. 8 (space_order <= 16)")
        if self.stencil not in STENCILS:
            raise ValueError(f"unknown stencil {self.stencil!r}, expected one of {STENCILS}")
        if self.ndim not in (2, 3):
            raise NotImplementedError("the B200 step is 2D or 3D")
        for name in ("domain", "dirichlet"):
            mask = getattr(self, name)
            if mask is not None and tuple(mask.shape) != self.Nx_padded:
                raise ValueError(f"{name} mask {tuple(mask.shape)} != {self.Nx_padded}")
        if self.masked and self.space_order // 2 >= CELL_HELD:
            raise ValueError(f"space_order {self.space_order} overflows the 3-bit cell radius")
        if self.devices is not None and len(tuple(self.devices)) > 1:
            raise NotImplementedError("the scalar path runs on one GPU: devices=(0,)")
        self.comp_stride = int(np.prod(self.Nx_padded))
        self.node_rows = self.ndim
        self.field_shape = self.Nx_padded
        if self.comp_stride >= 2**31:
            raise ValueError(
                f"{self.comp_stride} nodes overflow the int32 flat index; coarsen the grid"
            )
        if min(self.Nx) < self.space_order // 2 + 3:
            raise ValueError(
                f"Nx {self.Nx} cannot mirror the taps of space_order {self.space_order}: "
                f"at least {self.space_order // 2 + 3} nodes an axis"
            )
        if self.pml is not None:
            validate_pml(self)
        self._plan = None

    # ------------------------------------------------------------------ helpers
    @property
    def masked(self) -> bool:
        return self.domain is not None or self.dirichlet is not None

    @property
    def radius(self) -> int:
        return self.space_order // 2

    @property
    def reach(self) -> int:
        """Nodes one step reads past a point (cuwave wave.py:542-545)."""
        return self.space_order // 2

    def adjoint_mass_factor(self) -> float:
        """1 / dt^2, the residual's own scale (cuwave wave.py:597-599)."""
        return 1.0 / self.dt**2

    def pml_slabs(self) -> list[tuple]:
        """(d, lo, hi, profile) per lined axis (cuwave wave.py:587-595)."""
        if self.pml is None:
            return []
        widths, profiles = pml_widths(self), pml_profiles(self)
        return [
            (d, lo, hi, profile)
            for d, ((lo, hi), profile) in enumerate(zip(widths, profiles))
            if profile is not None
        ]

    def plan(self) -> nat.Plan:
        """The native plan of this configuration, made once."""
        if self._plan is None:
            grid = nat.Grid()
            grid.ndim = self.ndim
            for d, n in enumerate(self.Nx):
                grid.nx[d] = n
            grid.radius = self.radius
            grid.precision = 4 if self.precision == "float32" else 8
            for k, c in enumerate(operator_row(self.space_order, self.stencil)):
                grid.coeffs[k] = float(self.np_dtype(c))
            for d, f in enumerate(self.step_factors()):
                grid.factors[d] = float(f)
            grid.dt = float(self.dt)
            grid.dirichlet = face_mask(self, Dirichlet)
            grid.neumann = face_mask(self, Neumann)
            if self.pml is not None:
                for d, (lo, hi) in enumerate(pml_widths(self)):
                    grid.pml_lo[d], grid.pml_hi[d] = lo, hi
            self._plan = nat.Plan(grid)
        return self._plan

    def __getstate__(self):
        state = dict(self.__dict__)
        state["_plan"] = None
        return state


def mirror_ghosts(sim: Simulation, field: torch.Tensor) -> torch.Tensor:
    """Copy each face's second interior node onto its ghost, in place (cuwave wave.py:125-134)."""
    for d in range(sim.ndim):
        for ghost, mirror in ((0, 2), (sim.Nx[d] - 1, sim.Nx[d] - 3)):
            dst = [slice(None)] * sim.ndim
            dst[d] = ghost
            src = [slice(None)] * sim.ndim
            src[d] = mirror
            field[tuple(dst)] = field[tuple(src)]
    return field


def stepped_nodes(sim: Simulation) -> torch.Tensor:
    """The nodes the step updates: `domain` (all by default) less `dirichlet` (cuwave wave.py:665-672)."""
    stepped = torch.ones(sim.Nx_padded, dtype=torch.bool, device=device())
    if sim.domain is not None:
        stepped &= as_device(sim.domain, torch.bool)
    if sim.dirichlet is not None:
        stepped &= ~as_device(sim.dirichlet, torch.bool)
    return stepped


def domain_cells(sim: Simulation) -> torch.Tensor:
    """Per node of a masked grid, the radii of its two cells along each axis, packed
    (cuwave wave.py:675-726).

    A cell's taps may only reach stepped nodes (ghosts count as stepped), so each radius
    is capped by the run of stepped nodes on either side and by the box wall; a cell
    leaving the stepped set is closed (radius 0) unless the node across is held, which
    opens it onto a zero at its midpoint (CELL_HELD). The code is 0 for a node not
    stepped, CELL_DEEP where every radius is the full one, else
    (r_plus | r_minus << 3) << 6 d summed over the axes.
    """
    R = sim.radius
    dev = device()
    shape = sim.Nx_padded
    interior = tuple(slice(1, n - 1) for n in sim.Nx)
    inside = torch.ones(shape, dtype=torch.bool, device=dev)
    inside[interior] = stepped_nodes(sim)[interior]
    held = torch.zeros(shape, dtype=torch.bool, device=dev)
    if sim.dirichlet is not None:
        held[interior] = as_device(sim.dirichlet, torch.bool)[interior]

    def shifted(mask, d, k, fill):
        """mask[i + k] along axis d, `fill` past the array."""
        out = torch.full_like(mask, fill)
        n = shape[d]
        if abs(k) >= n:
            return out
        dst = [slice(None)] * sim.ndim
        src = [slice(None)] * sim.ndim
        dst[d] = slice(0, n - k) if k >= 0 else slice(-k, n)
        src[d] = slice(k, n) if k >= 0 else slice(0, n + k)
        out[tuple(dst)] = mask[tuple(src)]
        return out

    code = torch.zeros(shape, dtype=torch.int32, device=dev)
    deep = inside.clone()
    for d in range(sim.ndim):
        view = [1] * sim.ndim
        view[d] = -1
        a = torch.arange(shape[d], device=dev, dtype=torch.int32).reshape(view)
        wall = torch.clamp(torch.minimum(a, sim.Nx[d] - 1 - a), max=R)

        def run(sign):
            count = torch.zeros(shape, dtype=torch.int32, device=dev)
            on = torch.ones_like(inside)
            for k in range(1, R + 1):
                on &= shifted(inside, d, sign * k, True)
                count += (on & (k <= wall)).to(torch.int32)
            return count

        up, down = run(1), run(-1)
        rp = torch.minimum(wall, torch.minimum(1 + down, up))
        rm = torch.minimum(wall, torch.minimum(down, 1 + up))
        rp = torch.where((rp == 0) & shifted(held, d, 1, False), CELL_HELD, rp)
        rm = torch.where((rm == 0) & shifted(held, d, -1, False), CELL_HELD, rm)
        code |= (rp | (rm << 3)) << (6 * d)
        deep &= (rp == wall) & (rm == wall)
    code = torch.where(deep, CELL_DEEP, code)
    return torch.where(inside, code, 0).to(torch.int32).contiguous()


def require_stepped(sim: Simulation, position: torch.Tensor, what: str) -> None:
    """Raise for a point on a node a masked step never updates (cuwave wave.py:964-967)."""
    if not sim.masked or position.numel() == 0:
        return
    stepped = stepped_nodes(sim)
    if not bool(stepped[tuple(grid_rows(sim, position).long())].all()):
        raise ValueError(f"a {what} reaches a node that is never stepped")


def grid_coords(Nx, dx, dtype=torch.float64) -> list[torch.Tensor]:
    """Padded grid coordinates, node 1 at the origin (cuwave wave.py:137-143)."""
    dev = device()
    axes = [
        (torch.arange(n, dtype=dtype, device=dev) - 1) * d for n, d in zip(padded_shape(Nx), dx)
    ]
    return list(torch.meshgrid(*axes, indexing="ij"))


def apply_cell_weights(sim: Simulation, field: torch.Tensor) -> torch.Tensor:
    """In-place multiply by the cell weights W: 1/2 per wall (cuwave wave.py:336-344)."""
    for d in range(sim.ndim):
        for index in (1, sim.Nx[d] - 2):
            face = [slice(None)] * sim.ndim
            face[d] = index
            field[tuple(face)] *= 0.5
    return field


def grid_rows(sim: Simulation, position: torch.Tensor) -> torch.Tensor:
    return position[-sim.ndim :]


def sensor_cell_weights(sim: Simulation, sensors: torch.Tensor) -> torch.Tensor:
    """W at the sensor nodes (cuwave wave.py:347-354)."""
    rows = grid_rows(sim, sensors)
    w = torch.ones(sensors.shape[1], dtype=sim.dtype, device=sensors.device)
    for d in range(sim.ndim):
        for index in (1, sim.Nx[d] - 2):
            w = torch.where(rows[d] == index, w * 0.5, w)
    return w


def as_position(sim: Simulation, position) -> torch.Tensor:
    pos = as_device(position, torch.int32)
    if pos.dim() != 2 or pos.shape[0] != sim.node_rows:
        raise ValueError(
            f"position needs {sim.node_rows} rows in {sim.ndim}D, not {tuple(pos.shape)}"
        )
    if pos.numel():
        # every node a kernel reads or writes through a flat index must be on the grid
        lo = pos.amin(dim=1).cpu()
        hi = pos.amax(dim=1).cpu()
        for d in range(sim.ndim):
            if int(lo[d]) < 0 or int(hi[d]) > sim.Nx[d] - 1:
                raise ValueError(
                    f"position off the grid on axis {d}: [{int(lo[d])}, {int(hi[d])}] "
                    f"outside [0, {sim.Nx[d] - 1}]"
                )
    return pos


def flatten_indices(sim: Simulation, position) -> torch.Tensor:
    """(ndim, num) grid indices as int32 flat indices of the padded grid (cuwave wave.py:364-382)."""
    pos = as_position(sim, position)
    lin = torch.zeros(pos.shape[1], dtype=torch.int32, device=pos.device)
    for d in range(sim.ndim):
        lin += pos[d] * sim.strides[d]
    return lin


def narrow(values: torch.Tensor, dtype) -> torch.Tensor:
    """`values` stored as `dtype`, rounded to nearest even bfloat16 bits for BFLOAT16 (cuwave wave.py:848-853)."""
    if dtype != BFLOAT16:
        return values.to(dtype)
    bits = values.to(torch.float32).contiguous().view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    return ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16).to(torch.int32).to(torch.uint16)


def widen(values: torch.Tensor, dtype) -> torch.Tensor:
    """Inverse of `narrow` (cuwave wave.py:856-860)."""
    if values.dtype != BFLOAT16:
        return values.to(dtype)
    bits = values.to(torch.int32) << 16
    return bits.view(torch.float32).to(dtype)


# -------------------------------------------------------------------- the forward march
def require_off_held_walls(sim: Simulation, position: torch.Tensor) -> None:
    """Raise for a source on a Dirichlet wall node, held at zero (cuwave boundary.py:96-105)."""
    rows = grid_rows(sim, position)
    for face in faces_with(sim, Dirichlet):
        d, side = divmod(face, 2)
        wall = sim.Nx[d] - 2 if side else 1
        if bool((rows[d] == wall).any()):
            raise ValueError(f"a source on the wall node {wall} of Dirichlet face {face}, held at zero")


@dataclass
class Shot:
    """A source ready for the kernels: flat indices, weights and the (N, num) signal."""

    position: torch.Tensor
    lin: torch.Tensor
    weight: torch.Tensor
    signal: torch.Tensor
    foldable: bool = field(default=True)

    def points(self, row_add: int = 0, row_mul: int = 1) -> nat.Points:
        return nat.points(self.lin, self.signal, weight=self.weight, row_mul=row_mul,
                          row_add=row_add)


def prepare_shot(sim: Simulation, mat: dict, position, signal, weight=None) -> Shot:
    """Flatten a source and check its signal; `weight` defaults to the excitation weights."""
    pos = as_position(sim, position)
    sig = as_device(signal, sim.dtype)
    if sig.dim() != 2 or sig.shape[1] != pos.shape[1]:
        raise ValueError(f"signal {tuple(sig.shape)} does not match {pos.shape[1]} points")
    lin = flatten_indices(sim, pos)
    w = sim.excitation_weights(mat, lin) if weight is None else as_device(weight, sim.dtype)
    upper = torch.tensor(sim.Nx, device=pos.device, dtype=torch.int32)[:, None] - 2
    inner = bool(((pos >= 1) & (pos <= upper)).all()) if pos.shape[1] else True
    return Shot(pos, lin, w.contiguous(), sig.contiguous(), inner)


def forward_ops(sim: Simulation, mat: dict, a: nat.Level, b: nat.Level, c: nat.Level,
                shot: Shot | None, memory: list, *, records=(), replay=None,
                source_row: tuple[int, int] = (1, 0), fold: bool = True) -> list[nat.Op]:
    """The op list of one forward step c = step(a, b) in the reference's order.

    fd (+ pml) -> excitation -> [replay] -> refill -> records (cuwave wave.py:1119-1127):
    with the sources on interior nodes and nothing to replay, the excitation and the
    refill ride in the step kernel. `records` are (lin, record, row_mul, row_add,
    store) tuples written after the refill.
    """
    material = sim.material(mat)
    folded = fold and replay is None and (shot is None or shot.foldable) and not sim.masked
    flags = (nat.PML if sim.pml is not None else 0)
    mul, add = source_row
    src = shot.points(row_add=add, row_mul=mul) if shot is not None else nat.points(None, None)
    if folded:
        flags |= nat.FOLD_REFILL | (nat.FOLD_SOURCES if src.num else 0)
    ops = [nat.op(nat.OP_STEP, flags=flags, a=a, b=b, c=c, mat=material,
                  points=src if folded else nat.points(None, None), memory=memory)]
    if not folded:
        if src.num:
            ops.append(nat.op(nat.OP_EXCITE, a=c, points=src))
        if replay is not None:
            ops.append(nat.op(nat.OP_REPLAY, a=c, points=replay))
        ops.append(nat.op(nat.OP_REFILL, a=c))
    for lin, record, row_mul, row_add, store in records:
        pts = nat.points(lin, record, row_mul=row_mul, row_add=row_add, store=store)
        if pts.num:
            ops.append(nat.op(nat.OP_RECORD, a=c, points=pts))
    return ops


def pml_memory(sim: Simulation, rows: int, dev: torch.device) -> list:
    """Zeroed pml memory per axis: `rows` slab rows of every lined axis, None elsewhere."""
    plan = sim.plan()
    memory = [None, None, None]
    if sim.pml is not None:
        for d, *_ in sim.pml_slabs():
            memory[d] = torch.zeros((rows, plan.pml_row(d)), dtype=sim.dtype, device=dev)
    return memory


def simulate(sim: Simulation, source: Source, indicator, sensors=None, record_every=None,
             *, _mat: dict | None = None):
    """Run `sim` forward under `source` and material `indicator` (cuwave wave.py:1071-1163).

    Returns the final field over the logical grid (ghosts kept, the padding dropped), a
    view of the march's own slot, followed by the (N, num_sensors) record when `sensors`
    is given and the stacked host snapshots of the field every `record_every` steps.
    (`_mat` replaces the materials built from `indicator`.)
    """
    dev = device()
    mat = sim.build_materials(indicator) if _mat is None else _mat
    shot = prepare_shot(sim, mat, source.position, source.signal)
    require_off_held_walls(sim, shot.position)
    require_stepped(sim, shot.position, "source")
    if shot.signal.shape[0] < sim.N:
        raise ValueError(f"the signal has {shot.signal.shape[0]} rows for {sim.N} steps")
    plan = sim.plan()
    U = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
    memory = pml_memory(sim, 3, dev)
    records = []
    um = None
    if sensors is not None:
        require_stepped(sim, as_position(sim, sensors), "sensor")
        sensor_lin = flatten_indices(sim, sensors)
        um = torch.zeros((sim.N, sensor_lin.numel()), dtype=sim.dtype, device=dev)
        records.append((sensor_lin, um, 1, 0, nat.STORE_NATIVE))
    # U[t % 2] takes u^t over u^(t - 2), so the rotation is a function of t alone
    ops = forward_ops(
        sim, mat, nat.level(U, add=0, period=2), nat.level(U, add=1, period=2),
        nat.level(U, add=0, period=2), shot, memory, records=records,
    )
    interior = (Ellipsis, *(slice(0, n) for n in sim.Nx))
    snapshots = []
    if record_every is None:
        plan.march(ops, 0, sim.N)
    else:
        t = 0
        while t < sim.N:
            stop = min(sim.N, (t + record_every - 1) // record_every * record_every + 1)
            plan.march(ops, t, stop - t)
            if (stop - 1) % record_every == 0:
                snapshots.append(U[(stop - 1) % 2][interior].cpu().numpy())
            t = stop
    out = (U[(sim.N - 1) % 2][interior],)
    if sensors is not None:
        out += (um,)
    if record_every is not None:
        out += (np.stack(snapshots),)
    return out if len(out) > 1 else out[0]
