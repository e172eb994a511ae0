"""CPU ORACLE -- test infrastructure, not the product.

Only tests/, `__graft_entry__.smoke()` and bench.py's cpu_baseline leg import this, and
only as the checker the CUDA path is compared against. It restates cmpmech/cuwave's
scalar-wave path on the CPU: the kernels in oracle_impl.h (plain C, one function per
reference kernel launch) and, here in numpy, the setup and the drivers around them:

    cell coefficients      cuwave/stencils.py:11-58
    stable_dt              cuwave/wave.py:44-54
    pml profiles           cuwave/boundary.py:327-361
    materials              cuwave/scalar.py:407-415, 927-934 (+ wave.mirror_ghosts)
    excitation weights     cuwave/scalar.py:858-872
    simulate               cuwave/wave.py:1071-1163 (plain step order, 1119-1127)
    sensitivity            cuwave/sensitivity.py:384-497 (fused adjoint, 468-480)
    source_sensitivity     cuwave/sensitivity.py:1054-1111
    spectral               cuwave/sensitivity.py:295-380, 896-1051 (dft_kernel,
                           cuwave/kernels/common.cuh:506-518, restated in numpy)
    superposition          cuwave/sensitivity.py:753-893 (superposed_kernel /
                           frechet_kernel, cuwave/kernels/scalar_sensitivity.cu:353-385,
                           600-668, restated in numpy)

Pinned against the reference's own outputs: tests/golden/*.npz, produced by running
the reference package itself (tests/golden/make_golden.py).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "liboracle.so"


def build() -> Path:
    """Compile liboracle.so from oracle.c when it is missing or older than its sources."""
    sources = [HERE / "oracle.c", HERE / "oracle_impl.h"]
    if LIBRARY.exists() and all(LIBRARY.stat().st_mtime >= s.stat().st_mtime for s in sources):
        return LIBRARY
    cc = os.environ.get("ORACLE_CC", "gcc")
    tmp = LIBRARY.with_suffix(".tmp.so")
    cmd = [cc, "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
           str(HERE / "oracle.c"), "-o", str(tmp), "-lm"]
    done = subprocess.run(cmd, capture_output=True, text=True)
    if done.returncode:
        raise RuntimeError(f"{' '.join(cmd)} failed:\n{done.stderr}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


class Geo(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("ext", ctypes.c_int * 3),
        ("s", ctypes.c_int * 3),
        ("lo", ctypes.c_int * 3),
        ("hi", ctypes.c_int * 3),
        ("dir", ctypes.c_int),
        ("R", ctypes.c_int),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(build()))
        for sfx in ("_f32", "_f64"):
            getattr(_lib, "orc_slab_size" + sfx).restype = ctypes.c_long
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _r(dtype, v):
    return ctypes.c_float(v) if dtype == np.float32 else ctypes.c_double(v)


# ------------------------------------------------------------------------- setup
def cell_coefficients(radius: int, stencil: str = "taylor") -> np.ndarray:
    """Cell-flux weights w_1..w_R (cuwave stencils.py:11-58)."""
    if stencil == "taylor":
        x = np.arange(-radius, radius + 1)
        A = x[None, :] ** np.arange(2 * radius + 1)[:, None]
        rhs = np.zeros(2 * radius + 1)
        rhs[2] = 2.0
        w = np.linalg.solve(A, rhs)
        return np.array([w[radius + 1 + k:].sum() for k in range(radius)])
    k = np.arange(1, radius + 1)
    for band in np.linspace(np.pi, 0.0, 400, endpoint=False):
        theta = np.linspace(band / 400, band, 400)
        G = 2.0 * np.sin(np.outer(theta, k - 0.5)) / theta[:, None]
        G *= 2.0 * np.sin(theta / 2.0)[:, None] / theta[:, None]
        cons = (2 * k - 1.0)[None]
        K = np.block([[G.T @ G, cons.T], [cons, np.zeros((1, 1))]])
        c = np.linalg.solve(K, np.append(G.sum(axis=0), 1.0))[:radius]
        if np.abs(np.sqrt(G @ c) - 1.0).max() <= 1e-3:
            return c
    raise ValueError(radius)


def stable_dt(dx, wavespeed, space_order=2, stencil="optimized") -> float:
    c = cell_coefficients(space_order // 2, stencil)
    lam = 4.0 * abs(float(c @ (-1.0) ** np.arange(len(c))))
    return 2.0 / (wavespeed * float(np.sqrt(lam * sum(1.0 / d**2 for d in dx))))


def padded(Nx):
    return (*Nx[:-1], (Nx[-1] + 31) // 32 * 32)


def mirror_ghosts(Nx, f):
    for d in range(len(Nx)):
        for ghost, mirror in ((0, 2), (Nx[d] - 1, Nx[d] - 3)):
            dst = [slice(None)] * len(Nx)
            src = [slice(None)] * len(Nx)
            dst[d], src[d] = ghost, mirror
            f[tuple(dst)] = f[tuple(src)]
    return f


def pml_profiles(Nx, dx, dt, widths, width, wavespeed, reflection, frequency, dtype):
    """(4, Nx[d]) a_node, b_node, a_half, b_half per lined axis (cuwave boundary.py:327-361)."""
    L = width - 1
    out = []
    for d, (lo, hi) in enumerate(widths):
        if not lo + hi:
            out.append(None)
            continue
        n = Nx[d]
        damping = -3.0 * wavespeed * np.log(reflection) / (2.0 * L * dx[d])
        rows = []
        for shift in (0.0, 0.5):
            position = np.arange(n) + shift
            distance = np.full(n, np.inf)
            if lo:
                distance = np.minimum(distance, np.abs(position - 1))
            if hi:
                distance = np.minimum(distance, np.abs(n - 2 - position))
            depth = np.clip((L - distance) / L, 0.0, 1.0)
            d0 = damping * depth**2
            alpha = np.pi * frequency
            inside = depth > 0.0
            b = np.where(inside, np.exp(-(d0 + alpha) * dt), 1.0)
            a = np.where(inside, d0 / np.maximum(d0 + alpha, 1e-300) * (b - 1.0), 0.0)
            rows += [a, b]
        out.append(np.ascontiguousarray(np.stack(rows).astype(dtype)))
    return out


def cell_table(radius: int, stencil: str, dtype) -> np.ndarray:
    """(R, R) rows OP_W(r, 1..r): Taylor below R, `stencil` at R (cuwave stencils.py:186-196)."""
    table = np.zeros((radius, radius))
    for r in range(1, radius + 1):
        table[r - 1, :r] = cell_coefficients(r, stencil if r == radius else "taylor")
    if radius == 1:
        table[0, 0] = 1.0  # OP_W is the literal 1 at radius 1 (common.cuh:25-27)
    return table.astype(dtype)


def domain_cells(Nx, R, stepped, held=None):
    """Cell codes of a masked domain over the padded grid (cuwave wave.py:675-726): 0 not
    stepped, 1 << 30 all cells at the full radius, else the packed radii per axis."""
    shape = padded(Nx)
    ndim = len(Nx)
    interior = tuple(slice(1, n - 1) for n in Nx)
    inside = np.ones(shape, bool)
    inside[interior] = np.asarray(stepped, bool)[interior]
    hold = np.zeros(shape, bool)
    if held is not None:
        hold[interior] = np.asarray(held, bool)[interior]

    def moved(mask, d, k, fill):
        padded_ = np.pad(mask, R, constant_values=fill)
        window = [slice(R, R + n) for n in shape]
        window[d] = slice(R + k, R + k + shape[d])
        return padded_[tuple(window)]

    code = np.zeros(shape, np.int64)
    deep = inside.copy()
    for d in range(ndim):
        view = [1] * ndim
        view[d] = -1
        a = np.arange(shape[d]).reshape(view)
        wall = np.minimum(R, np.minimum(a, Nx[d] - 1 - a))
        runs = []
        for sign in (1, -1):
            count = np.zeros(shape, np.int64)
            on = np.ones(shape, bool)
            for k in range(1, R + 1):
                on &= moved(inside, d, sign * k, True)
                count += on & (k <= wall)
            runs.append(count)
        up, down = runs
        rp = np.minimum(wall, np.minimum(1 + down, up))
        rm = np.minimum(wall, np.minimum(down, 1 + up))
        rp = np.where((rp == 0) & moved(hold, d, 1, False), 7, rp)
        rm = np.where((rm == 0) & moved(hold, d, -1, False), 7, rm)
        code |= (rp | rm << 3) << (6 * d)
        deep &= (rp == wall) & (rm == wall)
    code = np.where(deep, 1 << 30, code)
    return np.where(inside, code, 0).astype(np.int32)


def acoustic_materials(Nx, indicator, rho1, rho2, kappa1, kappa2, dtype):
    """(stiff, minv) of AcousticWave, ghosts mirrored (cuwave scalar.py:927-934, 407-415)."""
    ind = np.asarray(indicator, dtype=dtype)
    rho_inv = dtype(1 / rho1) + ind * dtype(1 / rho2 - 1 / rho1)
    kappa_inv = dtype(1 / kappa1) + ind * dtype(1 / kappa2 - 1 / kappa1)
    minv = dtype(1) / kappa_inv
    return mirror_ghosts(Nx, rho_inv.astype(dtype)), mirror_ghosts(Nx, minv.astype(dtype))


@dataclass
class Case:
    """One configuration of the scalar step and its inputs, all numpy."""

    Nx: tuple
    R: int
    coeffs: np.ndarray        # w_1..w_R (float64; rounded to dtype on use)
    factors: tuple            # f_d
    dt: float
    stiff: np.ndarray         # padded grid
    minv: np.ndarray | None   # padded grid, None to derive 1 / stiff
    dtype: type = np.float32
    dirichlet: int = 0
    neumann: int | None = None
    damping: np.ndarray | None = None
    widths: tuple | None = None   # ((lo, hi),) per axis of a pml
    profiles: list | None = None  # per axis (4, Nx[d]) or None
    source_lin: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    source_weight: np.ndarray | None = None
    signal: np.ndarray | None = None   # (N, nsrc)
    sensor_lin: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    cells: np.ndarray | None = None    # a masked domain's cell codes (domain_cells)
    table: np.ndarray | None = None    # with cells: (R, R) OP_W rows (cell_table)

    def __post_init__(self):
        self.ndim = len(self.Nx)
        self.shape = padded(self.Nx)
        if self.neumann is None:
            self.neumann = ((1 << (2 * self.ndim)) - 1) & ~self.dirichlet
        g = Geo()
        g.ndim = self.ndim
        strides = [1] * self.ndim
        for d in range(self.ndim - 2, -1, -1):
            strides[d] = strides[d + 1] * self.shape[d + 1]
        for d in range(self.ndim):
            g.n[d], g.ext[d], g.s[d] = self.Nx[d], self.shape[d], strides[d]
            if self.widths is not None:
                g.lo[d], g.hi[d] = self.widths[d]
        g.dir = self.dirichlet
        g.R = self.R
        self.geo = g
        self.strides = strides
        self.sfx = "_f32" if self.dtype == np.float32 else "_f64"
        self.w = np.zeros(8, self.dtype)
        self.w[: self.R] = np.asarray(self.coeffs, np.float64).astype(self.dtype)
        self.f = np.zeros(3, self.dtype)
        self.f[: self.ndim] = np.asarray(self.factors, self.dtype)
        self.derive = self.minv is None

    def fn(self, name):
        return getattr(lib(), name + self.sfx)

    def slab_size(self, d):
        return int(self.fn("orc_slab_size")(ctypes.byref(self.geo), d))

    def lined(self):
        return [d for d in range(self.ndim) if self.widths is not None and sum(self.widths[d])]

    def excitation_weights(self, lin):
        """dt^2 minv (/ (1 + beta)) at lin (cuwave scalar.py:858-872), source factor 1."""
        field_ = self.stiff if self.derive else self.minv
        w = field_.ravel()[lin]
        if self.derive:
            w = self.dtype(1) / w
        if self.damping is not None:
            beta = self.dtype(0.5) * w * self.damping.ravel()[lin] * self.dtype(self.dt)
            w = w / (self.dtype(1) + beta)
        return (self.dtype(self.dt**2) * w).astype(self.dtype)

    # ------------------------------------------------------------ single launches
    def step(self, u0, u1, u2):
        if self.cells is not None:
            # held in locals so the buffers outlive the call
            table = np.ascontiguousarray(self.table, self.dtype)
            cells = np.ascontiguousarray(self.cells, np.int32)
            self.fn("orc_step_cells")(
                ctypes.byref(self.geo), _p(self.w), _p(self.f), _r(self.dtype, self.dt),
                _p(u0), _p(u1), _p(u2), _p(self.stiff), _p(self.minv), _p(self.damping),
                int(self.derive), _p(cells), _p(table))
            return
        self.fn("orc_step")(ctypes.byref(self.geo), _p(self.w), _p(self.f), _r(self.dtype, self.dt),
                            _p(u0), _p(u1), _p(u2), _p(self.stiff), _p(self.minv),
                            _p(self.damping), int(self.derive))

    def pml(self, u1, u2, memory):
        for d in self.lined():
            self.fn("orc_pml")(ctypes.byref(self.geo), _p(self.w), d, _r(self.dtype, self.f[d]),
                               _p(u1), _p(u2), _p(self.stiff), _p(self.minv), int(self.derive),
                               _p(memory[d]), _p(self.profiles[d]))

    def excite(self, u, lin, weight, row):
        row = np.ascontiguousarray(row, self.dtype)
        self.fn("orc_excite")(_p(u), _p(lin), _p(weight), _p(row), int(lin.size))

    def refill(self, u):
        self.fn("orc_refill")(ctypes.byref(self.geo), _p(u), self.neumann, self.dirichlet)

    def memory(self):
        return {d: np.zeros((3, self.slab_size(d)), self.dtype) for d in self.lined()}

    # ------------------------------------------------------------------ drivers
    def forward(self, N, history=False):
        """N plain steps: fd, pml, excitation, refill, record (cuwave wave.py:1118-1127).

        Returns (final field, (N, nsens) traces) and, with `history`, the (N + 2) levels
        V with V[t + 2] = u^t as `sensitivity` stores them.
        """
        U = np.zeros((2, *self.shape), self.dtype)
        V = np.zeros((N + 2, *self.shape), self.dtype) if history else None
        mem = self.memory()
        um = np.zeros((N, self.sensor_lin.size), self.dtype)
        for t in range(N):
            if history:
                u0, u1, u2 = V[t], V[t + 1], V[t + 2]
            else:
                u0, u1, u2 = U[t % 2], U[1 - t % 2], U[t % 2]
            self.step(u0, u1, u2)
            self.pml(u1, u2, mem)
            if self.source_lin.size:
                self.excite(u2, self.source_lin, self.source_weight, self.signal[t])
            self.refill(u2)
            um[t] = u2.ravel()[self.sensor_lin]
        final = V[N + 1] if history else U[(N - 1) % 2]
        return (final, um, V) if history else (final, um)

    def cell_weights(self, field_):
        for d in range(self.ndim):
            for index in (1, self.Nx[d] - 2):
                face = [slice(None)] * self.ndim
                face[d] = index
                field_[tuple(face)] *= self.dtype(0.5)
        return field_

    def sensor_weights(self, lin):
        """W at flat indices lin (cuwave wave.py:347-354)."""
        w = np.ones(lin.size, self.dtype)
        rest = lin.astype(np.int64)
        coords = []
        for d in range(self.ndim):
            coords.append(rest // self.strides[d])
            rest = rest - coords[-1] * self.strides[d]
        for d in range(self.ndim):
            for index in (1, self.Nx[d] - 2):
                w = np.where(coords[d] == index, w * self.dtype(0.5), w)
        return w

    def pml_nodes(self):
        inside = np.zeros(self.shape, bool)
        for d in self.lined():
            lo, hi = self.widths[d]
            index = [slice(None)] * self.ndim
            for rows in (slice(1, 1 + lo), slice(self.Nx[d] - 1 - hi, self.Nx[d] - 1)):
                index[d] = rows
                inside[tuple(index)] = True
        interior = np.zeros(self.shape, bool)
        interior[tuple(slice(1, n - 1) for n in self.Nx)] = True
        return inside & interior

    def adjoint_signal(self, dphi):
        """dphi reversed over W (source factor 1) (cuwave sensitivity.py:272-292)."""
        return np.ascontiguousarray(
            np.asarray(dphi, self.dtype)[::-1] / self.sensor_weights(self.sensor_lin), self.dtype
        )

    def sensitivity(self, N, dphi_of):
        """Fused adjoint with stored history (cuwave sensitivity.py:384-497).

        `dphi_of(traces) -> (cost, dphi)`. Returns cost, {"mass", "stiff"}, traces.
        """
        _, um, V = self.forward(N, history=True)
        cost, dphi = dphi_of(um)
        signal = self.adjoint_signal(dphi)
        weight = self.excitation_weights(self.sensor_lin)
        g_mass = np.zeros(self.shape, self.dtype)
        g_stiff = np.zeros(self.shape, self.dtype)
        P = np.zeros((2, *self.shape), self.dtype)
        eta = {d: np.zeros((3, self.slab_size(d)), self.dtype) for d in self.lined()}
        mf = self.dtype(1.0 / self.dt**2)
        geo = ctypes.byref(self.geo)
        for m in range(N):
            l0, l1 = P[m % 2], P[1 - m % 2]
            u1 = V[N + 1 - m]
            self.fn("orc_adjoint")(geo, _p(self.w), _p(self.f), _r(self.dtype, self.dt), _p(l0),
                                   _p(l1), _p(l0), _p(u1), _p(g_mass), _p(g_stiff),
                                   _p(self.stiff), _p(self.minv), _p(self.damping),
                                   int(self.derive), _r(self.dtype, mf), 1)
            for d in self.lined():
                self.fn("orc_pml_aux")(geo, d, _r(self.dtype, self.f[d]), _p(l1), _p(self.stiff),
                                       _p(eta[d]), _p(self.profiles[d]))
                self.fn("orc_pml_adjoint")(geo, _p(self.w), d, _r(self.dtype, self.f[d]), _p(l0),
                                           _p(g_mass), _p(u1), _r(self.dtype, mf), 1,
                                           _p(self.stiff), _p(self.minv), int(self.derive),
                                           _p(eta[d]), _p(self.profiles[d]))
            row = np.ascontiguousarray(signal[m])
            self.fn("orc_load")(_p(l0), _p(self.sensor_lin), _p(weight), _p(row),
                                int(self.sensor_lin.size), _p(g_mass), _p(u1),
                                _r(self.dtype, mf))
        grads = {"mass": self.cell_weights(g_mass), "stiff": self.cell_weights(g_stiff)}
        layer = self.pml_nodes()
        for g in grads.values():
            g[layer] = 0
        return cost, grads, um

    def source_sensitivity(self, N, dphi_of):
        """d(cost)/d(signal) (cuwave sensitivity.py:1054-1111); source factor 1."""
        _, um = self.forward(N)
        cost, dphi = dphi_of(um)
        signal = self.adjoint_signal(dphi)
        weight = self.excitation_weights(self.sensor_lin)
        P = np.zeros((2, *self.shape), self.dtype)
        eta = {d: np.zeros((3, self.slab_size(d)), self.dtype) for d in self.lined()}
        lam = np.zeros((N, self.source_lin.size), self.dtype)
        geo = ctypes.byref(self.geo)
        if self.cells is not None:
            # a masked domain is stepped backwards by its own graded step (scalar.py:322-324)
            for m in range(N):
                l0, l1 = P[m % 2], P[1 - m % 2]
                self.step(l0, l1, l0)
                self.excite(l0, self.sensor_lin, weight, signal[m])
                self.refill(l0)
                lam[m] = l0.ravel()[self.source_lin]
            gradient = lam[::-1] * self.sensor_weights(self.source_lin)
            return cost, np.ascontiguousarray(gradient), um
        for m in range(N):
            l0, l1 = P[m % 2], P[1 - m % 2]
            self.fn("orc_adjoint")(geo, _p(self.w), _p(self.f), _r(self.dtype, self.dt), _p(l0),
                                   _p(l1), _p(l0), None, None, None, _p(self.stiff),
                                   _p(self.minv), _p(self.damping), int(self.derive),
                                   _r(self.dtype, 0.0), 0)
            for d in self.lined():
                self.fn("orc_pml_aux")(geo, d, _r(self.dtype, self.f[d]), _p(l1), _p(self.stiff),
                                       _p(eta[d]), _p(self.profiles[d]))
                self.fn("orc_pml_adjoint")(geo, _p(self.w), d, _r(self.dtype, self.f[d]), _p(l0),
                                           None, None, _r(self.dtype, 0.0), 0, _p(self.stiff),
                                           _p(self.minv), int(self.derive), _p(eta[d]),
                                           _p(self.profiles[d]))
            self.excite(l0, self.sensor_lin, weight, signal[m])
            self.refill(l0)
            lam[m] = l0.ravel()[self.source_lin]
        gradient = lam[::-1] * self.sensor_weights(self.source_lin)
        return cost, np.ascontiguousarray(gradient), um


    # ------------------------------------------------------------ superposition
    def densities(self, acc_mass, acc_stiff, before, middle, newest, ft, F):
        """Both Frechet densities of one triplet over the interior, in place.

        acc_mass += ft (newest - before)^2 and acc_stiff += sum_d F_d (middle[+s_d] -
        middle[-s_d])^2, each product rounded in the kernel's order (frechet_kernel,
        cuwave/kernels/scalar_sensitivity.cu:353-385; superposed_kernel 637-654 with
        newest = the middle level and before = the level it is about to overwrite).
        """
        dt_ = self.dtype
        inner = tuple(slice(1, n - 1) for n in self.Nx)
        dudt = newest[inner] - before[inner]
        acc_mass[inner] += (dt_(ft) * dudt) * dudt
        total = None
        for d in range(self.ndim):
            hi = tuple(slice(2, n) if e == d else slice(1, n - 1) for e, n in enumerate(self.Nx))
            lo = tuple(slice(0, n - 2) if e == d else slice(1, n - 1) for e, n in enumerate(self.Nx))
            g = middle[hi] - middle[lo]
            term = (dt_(F[d]) * g) * g
            total = term if total is None else total + term
        acc_stiff[inner] += total

    def superposed(self, u0, u1, u2, acc_mass, acc_stiff, ft, fs):
        """superposed_kernel (scalar_sensitivity.cu:600-668): the densities against u2's
        old value, then the plain step into u2."""
        dt_ = self.dtype
        # the kernel forms sum_d f_d g_d^2, then scales it by fs
        inner = tuple(slice(1, n - 1) for n in self.Nx)
        dudt = u1[inner] - u2[inner]
        acc_mass[inner] += (dt_(ft) * dudt) * dudt
        total = None
        for d in range(self.ndim):
            hi = tuple(slice(2, n) if e == d else slice(1, n - 1) for e, n in enumerate(self.Nx))
            lo = tuple(slice(0, n - 2) if e == d else slice(1, n - 1) for e, n in enumerate(self.Nx))
            g = u1[hi] - u1[lo]
            term = (self.f[d] * g) * g
            total = term if total is None else total + term
        acc_stiff[inner] += dt_(fs) * total
        self.step(u0, u1, u2)

    def superposition(self, N, dphi_of, scale=1.0, dx=None):
        """Gradients in three slots by superposition (cuwave sensitivity.py:753-893).

        Forward: the superposed step subtracts B(u, u) while it records; backward, the
        field runs back in time carrying w = u + k lambda (the source reversed and the
        adjoint load scaled by k, one step late) and adds B(w, w); the gradients are the
        difference over 2k, cell weighted. Returns cost, {"mass", "stiff"}, traces,
        cancellation.
        """
        dt_ = self.dtype
        dx = dx or (1.0,) * self.ndim
        U = np.zeros((3, *self.shape), dt_)
        um = np.zeros((N, self.sensor_lin.size), dt_)
        acc = {"mass": np.zeros(self.shape, dt_), "stiff": np.zeros(self.shape, dt_)}

        def factors(sign):
            ratios = [-sign / (2.0 * d) ** 2 / float(f) for d, f in zip(dx, self.f[: self.ndim])]
            return dt_(sign / (2.0 * self.dt) ** 2), dt_(ratios[0])

        ft, fs = factors(-1.0)
        for t in range(N):
            u0, u1, u2 = U[t % 3], U[(t + 1) % 3], U[(t + 2) % 3]
            self.superposed(u0, u1, u2, acc["mass"], acc["stiff"], ft, fs)
            if self.source_lin.size:
                self.excite(u2, self.source_lin, self.source_weight, self.signal[t])
            self.refill(u2)
            um[t] = u2.ravel()[self.sensor_lin]
        t = N - 1
        self.densities(acc["mass"], acc["stiff"], U[t % 3], U[(t + 1) % 3], U[(t + 2) % 3],
                       ft, [0.0] * self.ndim)
        cost, dphi = dphi_of(um)
        before = np.sqrt(sum(float(np.linalg.norm(f)) ** 2 for f in acc.values()))

        # the adjoint load one step late and scaled by k, beside the source reversed
        signal = np.asarray(dphi, dt_)[::-1] / self.sensor_weights(self.sensor_lin)
        signal = np.concatenate((signal[1:], np.zeros_like(signal[:1])))
        signal = dt_(scale) * signal
        lin = np.concatenate((self.sensor_lin, self.source_lin)).astype(np.int32)
        rows = np.ascontiguousarray(
            np.concatenate((signal, self.signal[:N][::-1]), axis=1), dt_)
        weight = self.excitation_weights(lin)
        ft, fs = factors(1.0)
        for t in range(N):
            u0, u1, u2 = (U[(N + i - t) % 3] for i in (1, 0, 2))
            self.superposed(u0, u1, u2, acc["mass"], acc["stiff"], ft if t else dt_(0.0), fs)
            self.excite(u2, lin, weight, rows[t])
            self.refill(u2)
        self.densities(acc["mass"], acc["stiff"], U[2], U[1], U[0], ft, [0.0] * self.ndim)
        after = np.sqrt(sum(float(np.linalg.norm(f)) ** 2 for f in acc.values()))
        cancellation = before / after if after > 0.0 else float("inf")
        norm = dt_(1.0 / (2.0 * scale))
        for f in acc.values():
            self.cell_weights(f)
            f *= norm
        return cost, acc, um, cancellation


    # ----------------------------------------------------------------- spectral
    def gradient(self, u0, u1, u2, l1, g_mass, g_stiff):
        """gradient_kernel (scalar_sensitivity.cu:303-350) with F_d = f_d / dt^2."""
        F = np.zeros(3, self.dtype)
        F[: self.ndim] = [self.dtype(float(f) / self.dt**2) for f in self.f[: self.ndim]]
        self.fn("orc_gradient")(ctypes.byref(self.geo), _p(self.w), _p(F), _p(u0), _p(u1),
                                _p(u2), _p(l1), _p(g_mass), _p(g_stiff), _p(self.stiff),
                                _r(self.dtype, 1.0 / self.dt**2))

    def adjoint_run_step(self, l0, l1, eta):
        """The transposed step alone, pml memory included (scalar.py:318-344)."""
        geo = ctypes.byref(self.geo)
        self.fn("orc_adjoint")(geo, _p(self.w), _p(self.f), _r(self.dtype, self.dt), _p(l0),
                               _p(l1), _p(l0), None, None, None, _p(self.stiff),
                               _p(self.minv), _p(self.damping), int(self.derive),
                               _r(self.dtype, 0.0), 0)
        for d in self.lined():
            self.fn("orc_pml_aux")(geo, d, _r(self.dtype, self.f[d]), _p(l1), _p(self.stiff),
                                   _p(eta[d]), _p(self.profiles[d]))
            self.fn("orc_pml_adjoint")(geo, _p(self.w), d, _r(self.dtype, self.f[d]), _p(l0),
                                       None, None, _r(self.dtype, 0.0), 0, _p(self.stiff),
                                       _p(self.minv), int(self.derive), _p(eta[d]),
                                       _p(self.profiles[d]))

    def spectral(self, N, dphi_of, frequencies, region=None, reach=None):
        """Gradients of a spectral cost by two forward-in-time runs with running DFTs
        (cuwave sensitivity.py:896-1051). Returns cost, {"mass", "stiff"}, traces, info."""
        from scipy import ndimage

        dt_ = self.dtype
        freqs = np.atleast_1d(np.asarray(frequencies, np.float64))
        logical = np.zeros(self.shape, bool)
        logical[tuple(slice(0, n) for n in self.Nx)] = True
        region = logical if region is None else np.asarray(region, bool)
        square = ndimage.generate_binary_structure(self.ndim, self.ndim)
        reach = self.R if reach is None else reach
        kept = ndimage.binary_dilation(region, structure=square, iterations=reach + 1,
                                       brute_force=True)
        lin = np.flatnonzero(kept & logical).astype(np.int32)

        t = np.arange(N, dtype=np.float64) * self.dt
        phase = 2.0 * np.pi * t[:, None] * freqs[None, :]
        host = np.empty((N, 2 * len(freqs)))
        host[:, 0::2], host[:, 1::2] = np.cos(phase), -np.sin(phase)
        period = int(np.ceil(1.0 / (float(freqs.min()) * self.dt)))
        tail = host.copy()
        tail[: N - period] = 0.0
        table = np.concatenate((host, tail), axis=1).astype(dt_)
        F = len(freqs)

        U = np.zeros((2, *self.shape), dt_)
        mem = self.memory()
        um = np.zeros((N, self.sensor_lin.size), dt_)
        u_hat = np.zeros((4 * F, lin.size), dt_)
        for step in range(N):
            u0, u1 = U[step % 2], U[1 - step % 2]
            self.step(u0, u1, u0)
            self.pml(u1, u0, mem)
            if self.source_lin.size:
                self.excite(u0, self.source_lin, self.source_weight, self.signal[step])
            self.refill(u0)
            um[step] = u0.ravel()[self.sensor_lin]
            u_hat += table[step][:, None] * u0.ravel()[lin][None, :]
        u_last = U[(N - 1) % 2].ravel()[lin].astype(np.float64)
        cost, dphi = dphi_of(um)

        basis = np.empty_like(host)
        basis[:, 0::2], basis[:, 1::2] = host[:, 0::2], -host[:, 1::2]
        target = np.asarray(dphi).astype(np.float64)
        coef = np.linalg.lstsq(basis, target, rcond=None)[0]
        norm = float(np.linalg.norm(target))
        fit = float(np.linalg.norm(target - basis @ coef)) / norm if norm > 0.0 else 0.0
        load = coef[0::2] + 1j * coef[1::2]
        weights = self.sensor_weights(self.sensor_lin).astype(np.float64)
        sensor_weight = self.excitation_weights(self.sensor_lin)

        def settled_spectrum(acc, last, f):
            whole = acc[0].astype(np.complex128) + 1j * acc[1]
            late = acc[2].astype(np.complex128) + 1j * acc[3]
            z = np.exp(-2j * np.pi * f * self.dt)
            late = late - last * complex(np.sum(z ** np.arange(N - period, N)))
            n = float(np.linalg.norm(whole))
            share = float(np.linalg.norm(late)) / n if n > 0.0 else 0.0
            return whole + last * (z**N / (1.0 - z)), share

        g_mass = np.zeros(self.shape, dt_)
        g_stiff = np.zeros(self.shape, dt_)
        fields = np.zeros((4, *self.shape), dt_)
        decay = 0.0
        for k, f in enumerate(freqs):
            sigma = 1.0 / f
            if 8.0 * sigma > t[-1]:
                raise ValueError("the adjoint pulse is longer than the run")
            envelope = np.exp(-0.5 * ((t - 4.0 * sigma) / sigma) ** 2)
            omega = 2.0 * np.pi * f
            carriers = envelope * np.stack((np.cos(omega * t), np.sin(omega * t)))
            spec = carriers @ np.exp(-1j * omega * t)
            amplitudes = np.linalg.solve(np.array([spec.real, spec.imag]),
                                         np.stack((load[k].real, load[k].imag)))
            pulse = np.ascontiguousarray((carriers.T @ amplitudes) / weights, dt_)
            columns = [2 * k, 2 * k + 1, 2 * F + 2 * k, 2 * F + 2 * k + 1]
            ftable = table[:, columns]
            P = np.zeros((2, *self.shape), dt_)
            eta = {d: np.zeros((5, self.slab_size(d)), dt_) for d in self.lined()}
            lam_hat = np.zeros((4, lin.size), dt_)
            for step in range(N):
                l0, l1 = P[step % 2], P[1 - step % 2]
                self.adjoint_run_step(l0, l1, eta)
                self.excite(l0, self.sensor_lin, sensor_weight, pulse[step])
                self.refill(l0)
                lam_hat += ftable[step][:, None] * l0.ravel()[lin][None, :]
            lam_last = P[(N - 1) % 2].ravel()[lin].astype(np.float64)
            spectrum, share = settled_spectrum(u_hat[columns], u_last, f)
            adjoint_hat, adjoint_share = settled_spectrum(lam_hat, lam_last, f)
            decay = max(decay, share, adjoint_share)
            shift = np.exp(-2j * np.pi * f * self.dt)
            triplet = (spectrum * shift**2, spectrum * shift, spectrum)
            for part, sign in ((np.real, 1.0), (np.imag, -1.0)):
                for j, value in enumerate((*triplet, sign * adjoint_hat)):
                    fields[j].ravel()[lin] = part(value)
                self.gradient(fields[0], fields[1], fields[2], fields[3], g_mass, g_stiff)
        grads = {"mass": self.cell_weights(g_mass), "stiff": self.cell_weights(g_stiff)}
        layer = self.pml_nodes()
        for g in grads.values():
            g[layer] = 0
            g[~region] = 0.0
        return cost, grads, um, {"decay": decay, "fit": fit}


def l2(observed):
    """The least-squares objective (cuwave sensitivity.py:93-100)."""
    def objective(traces):
        residual = traces - observed
        return 0.5 * float(np.sum(residual**2)), residual
    return objective


# ------------------------------------------------------ the reference's own kernels
REF_DIR = HERE / "_ref"


def ref_library(ndim=3, radius=4, stencil="optimized", precision="float32") -> tuple[Path, str]:
    """(path, instruction-set level) of the reference's kernels built for this host by
    ref_build.py: the highest level the host's CPU supports."""
    import importlib.util
    import sys

    spec = importlib.util.spec_from_file_location("_oracle_ref_build", HERE / "ref_build.py")
    module = sys.modules.get(spec.name)
    if module is None:
        module = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = module
        spec.loader.exec_module(module)
    return module.library(ndim, radius, stencil, precision)


def ref_simulate(case: "Case", N: int, threads: int | None = None, library: Path | None = None):
    """The reference's own fd/pml/excitation/refill/record kernels (built by ref_build.py
    from its sources) stepped N times on a 2D or 3D Neumann case; returns (field, traces),
    the field over the padded grid. `library` names a build; by default the one for this
    host's instruction set."""
    ndim = len(case.Nx)
    path = library or ref_library(ndim, case.R, "optimized",
                                  "float32" if case.dtype == np.float32 else "float64")[0]
    if not path.exists():
        raise FileNotFoundError(f"{path.name} is not built: run oracle/ref_build.py")
    if threads is not None:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    lib = ctypes.CDLL(str(path))
    U = np.zeros((2, *case.shape), case.dtype)
    lo = hi = 0
    aux_parts, prof_parts = [], []
    if case.widths is not None:
        lo, hi = case.widths[0]
        for d in range(ndim):
            plane = int(np.prod([case.shape[e] for e in range(ndim) if e != d]))
            aux_parts.append(np.zeros(3 * (lo + hi) * plane, case.dtype))
            prof_parts.append(case.profiles[d].ravel())
    aux = np.concatenate(aux_parts) if aux_parts else np.zeros(1, case.dtype)
    prof = np.concatenate(prof_parts) if prof_parts else np.zeros(1, case.dtype)
    um = np.zeros((N, case.sensor_lin.size), case.dtype)
    f = np.zeros(3, case.dtype)
    f[:ndim] = case.f[:ndim]
    signal = np.ascontiguousarray(case.signal[:N], case.dtype)
    n = np.zeros(3, np.int32)
    n[:ndim] = case.Nx
    rc = lib.ref_simulate(
        _p(n), int(case.shape[-1]), _p(U), _p(case.stiff), _p(case.minv), int(case.derive), _p(f),
        lo, hi, _p(aux), _p(prof), _p(case.source_lin), _p(case.source_weight), _p(signal),
        int(case.source_lin.size), _p(case.sensor_lin), _p(um), int(case.sensor_lin.size), N,
    )
    if rc:
        raise RuntimeError("ref_simulate refused the case")
    return U[(N - 1) % 2], um
