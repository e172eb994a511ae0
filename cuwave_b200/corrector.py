"""A learned dispersion corrector: a 2x-coarser, lower-order grid standing in for the fine one.

The coarse solve (grid spacing 2 dx, space order 4, its own time step) disperses: its
waves run at slightly wrong speeds. Every `EVERY` coarse steps a small convolutional
network predicts, from the coarse field's two levels and the material, the difference
between the fine solve (restricted to the coarse nodes) and the coarse one, and the
correction is added to the coarse field. The network is trained on pairs the plain
solver makes (fine runs restricted to the coarse grid, coarse runs of `EVERY` steps from
them), forward and backward through the project's own BF16 tensor-core convolutions
(cwb_conv_bf16_fwd / cwb_conv_bf16_bwd: warp-level MMA, FP32 accumulation), with Adam on
FP32 master weights. `corrected_traces` runs the corrected coarse solve, and
`learned_or_fine` falls back to the fine solve when the corrector's own error estimate
(the size of its corrections against the field) exceeds a tolerance.

Layout: activations channels-last (batch, height, width, channels) over the coarse grid's
logical nodes; layers 4 -> 32 -> 32 -> 2 channels of 5x5 convolutions, ReLU between, the
input's fourth channel held at zero (the kernels take an even channel count). The two
outputs correct the coarse field's two levels, so the leapfrog's velocity is corrected
with its displacement. The coarse node i sits on the fine node 2 i - 1 (both grids put node 1
at the origin).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat
from .scalar import AcousticWave
from .stencils import stable_dt
from .wave import Source, device, flatten_indices, forward_ops, pml_memory, prepare_shot

EVERY = 8  # coarse steps between corrections
CHANNELS = (4, 32, 32, 2)


def pack(w: torch.Tensor) -> torch.Tensor:
    """(cout, cin, 5, 5) FP32 weights as the kernels read them: (cout, kpad) BF16,
    k = (5 ky + kx) cin + ci, zero past 25 cin."""
    cout, cin = w.shape[:2]
    kpad = (25 * cin + 15) // 16 * 16
    out = torch.zeros((cout, kpad), dtype=torch.bfloat16, device=w.device)
    out[:, : 25 * cin] = w.permute(0, 2, 3, 1).reshape(cout, 25 * cin).to(torch.bfloat16)
    return out


def pack_transposed(w: torch.Tensor) -> torch.Tensor:
    """The data gradient's weights: flipped in space, input and output swapped."""
    return pack(w.flip(2, 3).permute(1, 0, 2, 3).contiguous())


def unpack(dw: torch.Tensor, cin: int) -> torch.Tensor:
    """(cout, kpad) gradient back to (cout, cin, 5, 5)."""
    cout = dw.shape[0]
    return dw[:, : 25 * cin].reshape(cout, 5, 5, cin).permute(0, 3, 1, 2).contiguous()


class Corrector:
    """The network, its FP32 master weights and its Adam state."""

    def __init__(self, seed: int = 0, dev: torch.device | None = None):
        dev = dev or device()
        gen = torch.Generator().manual_seed(seed)
        self.w, self.b = [], []
        for cin, cout in zip(CHANNELS[:-1], CHANNELS[1:]):
            std = math.sqrt(2.0 / (25 * cin))
            w = torch.randn((cout, cin, 5, 5), generator=gen) * std
            self.w.append(w.to(dev))
            self.b.append(torch.zeros(cout, device=dev))
        self.w[-1] *= 0.1  # start near the uncorrected solve
        self._hold()
        self.m = [torch.zeros_like(p) for p in self.params()]
        self.v = [torch.zeros_like(p) for p in self.params()]
        self.steps = 0

    def params(self) -> list[torch.Tensor]:
        return self.w + self.b

    def _hold(self) -> None:
        """The padding input channel stays zero."""
        self.w[0][:, 3] = 0.0

    # -------------------------------------------------------------------- passes
    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x (B, H, W, 4) BF16 -> the (B, H, W, 2) FP32 output; keeps what backward needs."""
        B, H, W, _ = x.shape
        self._x = x
        self._packed = [pack(w) for w in self.w]
        acts = [x]
        for layer in range(len(self.w) - 1):
            y = torch.empty((B, H, W, CHANNELS[layer + 1]), dtype=torch.bfloat16, device=x.device)
            nat.conv_fwd(acts[-1], self._packed[layer], self.b[layer], y16=y, relu=True)
            acts.append(y)
        out = torch.empty((B, H, W, CHANNELS[-1]), dtype=torch.float32, device=x.device)
        nat.conv_fwd(acts[-1], self._packed[-1], self.b[-1], y32=out)
        self._acts = acts
        return out

    def backward(self, dout: torch.Tensor) -> list[torch.Tensor]:
        """dL/d(output) (B, H, W, 2) FP32 -> dL/d(params) in the order of `params`."""
        B, H, W, _ = dout.shape
        dy = dout.to(torch.bfloat16).contiguous()
        gw, gb = [None] * len(self.w), [None] * len(self.w)
        for layer in range(len(self.w) - 1, -1, -1):
            x = self._acts[layer]
            cin, cout = CHANNELS[layer], CHANNELS[layer + 1]
            dw = torch.zeros((cout, (25 * cin + 15) // 16 * 16), dtype=torch.float32, device=dout.device)
            db = torch.zeros(cout, dtype=torch.float32, device=dout.device)
            nat.conv_bwd(dy, x, dw, db)
            gw[layer], gb[layer] = unpack(dw, cin), db
            if layer > 0:
                dx = torch.empty((B, H, W, cin), dtype=torch.bfloat16, device=dout.device)
                nat.conv_fwd(dy, pack_transposed(self.w[layer]), None, y16=dx, mask=x)
                dy = dx
        gw[0][:, 3] = 0.0
        return gw + gb

    def adam(self, grads: list[torch.Tensor], lr: float, beta1=0.9, beta2=0.999, eps=1e-8) -> None:
        self.steps += 1
        for p, g, m, v in zip(self.params(), grads, self.m, self.v):
            m.mul_(beta1).add_(g, alpha=1 - beta1)
            v.mul_(beta2).addcmul_(g, g, value=1 - beta2)
            mh = m / (1 - beta1**self.steps)
            vh = v / (1 - beta2**self.steps)
            p.sub_(lr * mh / (vh.sqrt() + eps))
        self._hold()


# ---------------------------------------------------------------- the two grids
@dataclass
class GridPair:
    """A fine grid and the coarse grid of twice its spacing over the same square."""

    fine: AcousticWave
    coarse: AcousticWave
    ratio: int  # fine steps per coarse step


def grid_pair(coarse_nodes: int, dx: float, cmax: float, coarse_steps: int) -> GridPair:
    """Fine: order 8 at dx; coarse: order 4 at 2 dx, `coarse_nodes` a side (ghosts in),
    CFL 0.5 by its own stencil; the fine step an integer fraction of the coarse one."""
    Nc = coarse_nodes
    Nf = 2 * Nc - 3
    dtc = 0.5 * stable_dt((2 * dx, 2 * dx), cmax, 4)
    ratio = max(1, math.ceil(dtc / (0.5 * stable_dt((dx, dx), cmax, 8))))
    common = dict(rho1=1.0, rho2=1.0, kappa1=1.0, kappa2=1.0 / (cmax * cmax * 1.5))
    fine = AcousticWave(Nx=(Nf, Nf), dx=(dx, dx), N=coarse_steps * ratio, dt=dtc / ratio,
                        space_order=8, **common)
    coarse = AcousticWave(Nx=(Nc, Nc), dx=(2 * dx, 2 * dx), N=coarse_steps, dt=dtc,
                          space_order=4, **common)
    return GridPair(fine, coarse, ratio)


def design_for(sim: AcousticWave, c: np.ndarray) -> np.ndarray:
    """The indicator making minv = c^2 on `sim`'s padded grid (c over its logical nodes)."""
    full = np.ones(sim.Nx_padded)
    full[: c.shape[0], : c.shape[1]] = c
    return AcousticWave.indicator_for_speed(full, sim.kappa2).astype(sim.np_dtype)


def restrict(fine_field: torch.Tensor, Nc: int) -> torch.Tensor:
    """The fine field on the coarse nodes (coarse node i = fine node 2 i - 1), ghosts
    mirrored as a Neumann refill leaves them."""
    idx = (torch.arange(Nc, device=fine_field.device) * 2 - 1).clamp(0, 2 * Nc - 4)
    out = fine_field[idx][:, idx].clone()
    out[0], out[-1] = out[2], out[-3]
    out[:, 0], out[:, -1] = out[:, 2], out[:, -3]
    return out


def speed_field(rng: np.random.Generator, n: int, cmin=1.0, cmax=2.0) -> np.ndarray:
    """A smooth random speed model: Gaussian blobs, or layers, between cmin and cmax."""
    y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    if rng.random() < 0.5:
        out = np.zeros((n, n))
        for _ in range(6):
            cy, cx, s = rng.uniform(0, n), rng.uniform(0, n), rng.uniform(n / 12, n / 4)
            out += rng.uniform(-1, 1) * np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2 * s * s))
        out = (out - out.min()) / max(out.max() - out.min(), 1e-9)
    else:
        edges = np.sort(rng.uniform(0, n, 4))
        out = np.searchsorted(edges, y + 0.15 * n * np.sin(x * rng.uniform(0.01, 0.05))) / 4.0
    return cmin + (cmax - cmin) * out


# ----------------------------------------------------------------- the solves
class Stepper:
    """A forward march of one simulation whose two levels the caller may read and set."""

    def __init__(self, sim: AcousticWave, indicator: np.ndarray, source: Source | None = None,
                 sensors=None):
        self.sim = sim
        dev = device()
        self.mat = sim.build_materials(indicator)
        self.shot = None
        if source is not None:
            self.shot = prepare_shot(sim, self.mat, source.position, source.signal)
        self.U = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
        self.memory = pml_memory(sim, 3, dev)
        records = []
        self.traces = None
        if sensors is not None:
            lin = flatten_indices(sim, sensors)
            self.traces = torch.zeros((sim.N, lin.numel()), dtype=sim.dtype, device=dev)
            records.append((lin, self.traces, 1, 0, nat.STORE_NATIVE))
            self._lin = lin
        a = nat.level(self.U, add=0, period=2)
        self.ops = forward_ops(sim, self.mat, a, nat.level(self.U, add=1, period=2), a,
                               self.shot, self.memory, records=records)
        self.t = 0

    def march(self, steps: int) -> None:
        steps = min(steps, self.sim.N - self.t)
        if steps > 0:
            self.sim.plan().march(self.ops, self.t, steps)
            self.t += steps

    def levels(self) -> tuple[torch.Tensor, torch.Tensor]:
        """(u^(t-1), u^(t-2)): the newest level and the one before."""
        return self.U[(self.t - 1) % 2], self.U[self.t % 2]

    def set_levels(self, newest: torch.Tensor, before: torch.Tensor, t: int = 0) -> None:
        """Continue the march from two given levels as if `t` steps had been taken."""
        self.t = t
        n0, n1 = newest.shape
        self.U.zero_()
        # step t reads U[t % 2] as u^(t-2) and U[(t + 1) % 2] as u^(t-1)
        self.U[(t + 1) % 2, :n0, :n1] = newest
        self.U[t % 2, :n0, :n1] = before


def features(newest: torch.Tensor, before: torch.Tensor, c: torch.Tensor):
    """The network's input over the logical nodes (B, H, W, 4) BF16, and the field scale."""
    scale = newest.pow(2).mean(dim=(-2, -1), keepdim=True).sqrt().clamp(min=1e-30)
    x = torch.zeros((*newest.shape, 4), dtype=torch.bfloat16, device=newest.device)
    x[..., 0] = (newest / scale).to(torch.bfloat16)
    x[..., 1] = ((newest - before) / scale).to(torch.bfloat16)
    x[..., 2] = ((c - 1.5) * 2.0).to(torch.bfloat16)
    return x, scale


def pulse(pair: GridPair, sim) -> np.ndarray:
    """A Gaussian pulse sampled at `sim`'s steps, about 8 coarse cells a wavelength at
    the slowest speed."""
    freq = 1.0 / (8 * pair.coarse.dx[0])
    t = np.arange(sim.N) * sim.dt
    return np.exp(-(((t - 1.2 / freq) * freq * math.pi) ** 2))


def shot_sources(pair: GridPair, pos) -> tuple[Source, Source]:
    """(fine, coarse) point sources at coarse node `pos` (fine node 2 pos - 1), their
    signals over the cell volume as a point source's are."""
    fine = Source(np.array([[2 * pos[0] - 1], [2 * pos[1] - 1]], np.int32),
                  (pulse(pair, pair.fine) / np.prod(pair.fine.dx))[:, None])
    coarse = Source(np.array([[pos[0]], [pos[1]]], np.int32),
                    (pulse(pair, pair.coarse) / np.prod(pair.coarse.dx))[:, None])
    return fine, coarse


def training_pairs(pair: GridPair, rng: np.random.Generator, shots: int, windows: int):
    """(inputs (P, H, W, 4) BF16, targets (P, H, W, 2) FP32 in field scale): fine runs
    restricted to the coarse grid against coarse runs of EVERY steps from them, for both
    levels the coarse run ends on."""
    Nc = pair.coarse.Nx[0]
    inputs, targets = [], []
    for _ in range(shots):
        c = speed_field(rng, Nc)
        cf = np.kron(c, np.ones((2, 2)))[: pair.fine.Nx[0], : pair.fine.Nx[1]]
        fine_ind, coarse_ind = design_for(pair.fine, cf), design_for(pair.coarse, c)
        pos = rng.integers(Nc // 4, 3 * Nc // 4, size=2)
        fine_src, coarse_src = shot_sources(pair, pos)
        fine = Stepper(pair.fine, fine_ind, fine_src)
        coarse = Stepper(pair.coarse, coarse_ind, coarse_src)
        cdev = torch.as_tensor(c, dtype=torch.float32, device=device())
        # windows over the whole run, the source's own injection in the coarse ones
        slots = np.arange(EVERY, pair.coarse.N - EVERY - 2, EVERY + 1)  # windows apart
        starts = sorted(rng.choice(slots, min(windows, len(slots)), replace=False))
        for n in starts:
            # fine levels after n - 1 and n coarse steps, then after n + EVERY
            fine.march(pair.ratio * (n - 1) - fine.t)
            before = restrict(fine.levels()[0][: pair.fine.Nx[0], : pair.fine.Nx[1]], Nc)
            fine.march(pair.ratio)
            newest = restrict(fine.levels()[0][: pair.fine.Nx[0], : pair.fine.Nx[1]], Nc)
            fine.march(pair.ratio * (EVERY - 1))
            truth_old = restrict(fine.levels()[0][: pair.fine.Nx[0], : pair.fine.Nx[1]], Nc)
            fine.march(pair.ratio)
            truth = restrict(fine.levels()[0][: pair.fine.Nx[0], : pair.fine.Nx[1]], Nc)
            coarse.set_levels(newest, before, n)
            coarse.march(EVERY)
            c_new, c_old = coarse.levels()
            c_new, c_old = c_new[:Nc, :Nc], c_old[:Nc, :Nc]
            x, scale = features(c_new, c_old, cdev)
            inputs.append(x)
            targets.append(torch.stack([(truth - c_new) / scale, (truth_old - c_old) / scale],
                                       dim=-1).float())
    return torch.stack(inputs), torch.stack(targets)


def train(net: Corrector, inputs: torch.Tensor, targets: torch.Tensor, steps: int,
          batch: int = 8, lr: float = 1e-3, seed: int = 0) -> list[float]:
    """Adam on the mean squared error of the predicted correction; the loss per step."""
    gen = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    for _ in range(steps):
        pick = torch.randint(0, inputs.shape[0], (batch,), generator=gen).to(inputs.device)
        out = net.forward(inputs[pick].contiguous())
        err = out - targets[pick]
        losses.append(float(err.pow(2).mean()))
        net.adam(net.backward(2.0 * err / err.numel()), lr)
    return losses


def corrected_traces(pair: GridPair, net: Corrector | None, c: np.ndarray, source: Source,
                     sensors) -> tuple[torch.Tensor, float]:
    """The coarse solve's receiver traces with the network's correction every EVERY steps
    (none without a net), and the corrector's error estimate: the largest correction
    against the field it corrected."""
    Nc = pair.coarse.Nx[0]
    run = Stepper(pair.coarse, design_for(pair.coarse, c), source, sensors)
    cdev = torch.as_tensor(c, dtype=torch.float32, device=device())
    estimate = 0.0
    while run.t < pair.coarse.N:
        run.march(EVERY)
        if net is None or run.t >= pair.coarse.N:
            continue
        newest, before = run.levels()
        x, scale = features(newest[:Nc, :Nc], before[:Nc, :Nc], cdev)
        delta = net.forward(x[None])[0] * scale
        estimate = max(estimate,
                       float(delta[..., 0].norm() / newest[:Nc, :Nc].norm().clamp(min=1e-30)))
        newest[:Nc, :Nc] += delta[..., 0]
        before[:Nc, :Nc] += delta[..., 1]
    return run.traces, estimate


def fine_traces(pair: GridPair, c: np.ndarray, source: Source, sensors) -> torch.Tensor:
    """The fine solve's traces at the coarse times (every `ratio`-th fine step)."""
    cf = np.kron(c, np.ones((2, 2)))[: pair.fine.Nx[0], : pair.fine.Nx[1]]
    run = Stepper(pair.fine, design_for(pair.fine, cf), source, sensors)
    run.march(pair.fine.N)
    return run.traces[pair.ratio - 1 :: pair.ratio]


def learned_or_fine(pair: GridPair, net: Corrector, c, coarse_source: Source,
                    fine_source: Source, coarse_sensors, fine_sensors, tolerance: float):
    """The corrected coarse traces, or the fine ones where the corrector's estimate
    exceeds `tolerance` (the plain fine solve is the fallback). Returns (traces, used)
    with `used` "learned" or "fine"."""
    traces, estimate = corrected_traces(pair, net, c, coarse_source, coarse_sensors)
    if estimate <= tolerance:
        return traces, "learned"
    return fine_traces(pair, c, fine_source, fine_sensors), "fine"
