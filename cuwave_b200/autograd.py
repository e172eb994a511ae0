"""Receiver traces as a differentiable function of the wave speed and the source signal.

`traces = wave_traces(c, signal, problem)` runs the scalar forward (AcousticWave with
rho = 1, so the inverse inertia is c^2 and the stiffness is uniform) and records the
sensors; `traces.backward(...)` runs the adjoint march once and returns

    dL/dc      = dL/dm * dm/dc,  m = 1 / c^2, dm/dc = -2 / c^3,
    dL/dsignal = lambda at the sources, reversed, times the adjoint weights,

where dL/dm is the cell-weighted inertia gradient the reference's `sensitivity` returns as
grads["mass"] (cuwave sensitivity.py:384-497) and dL/dsignal is its `source_sensitivity`
(sensitivity.py:1054-1111). With mode "reconstruction" the backward pass rebuilds the
forward field backwards in time behind the recorded PML strip (checkpointed when
`checkpoints` is set), so its memory does not grow with the number of steps; with mode
"history" it stores the N + 2 levels.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from .sensitivity import reconstruction_sensitivity, sensitivity
from .wave import Simulation, Source, as_device, as_position, mirror_ghosts, simulate


@dataclass
class Problem:
    """What stays fixed while c and the signal vary: the simulation, the source
    positions and the sensors, and how the backward pass keeps the forward field."""

    sim: Simulation  # an AcousticWave (its rho/kappa constants are not read here)
    source_position: object  # (ndim, num_sources)
    sensors: object  # (ndim, num_sensors)
    mode: str = "reconstruction"  # or "history"
    checkpoints: int | None = None
    strip_dtype: str | None = None


def speed_materials(sim: Simulation, c: torch.Tensor) -> dict:
    """The material dict of a speed field: stiffness 1, inverse inertia c^2, ghosts mirrored."""
    c = as_device(c, sim.dtype)
    if tuple(c.shape) != sim.Nx_padded:
        raise ValueError(f"c has shape {tuple(c.shape)}, the padded grid is {sim.Nx_padded}")
    minv = mirror_ghosts(sim, (c * c).contiguous())
    stiff = torch.ones(sim.Nx_padded, dtype=sim.dtype, device=c.device)
    mat = {"stiff": stiff, "minv": minv, "damping": None, "profiles": [None] * 3,
           "uniform": True, "stiff_value": 1.0}
    if sim.damping is not None:
        mat["damping"] = as_device(sim.damping, sim.dtype)
    for d, lo, hi, profile in sim.pml_slabs():
        mat["profiles"][d] = torch.as_tensor(profile, device=c.device)
    return mat


class WaveTraces(torch.autograd.Function):
    """(c, signal) -> traces through the native forward and adjoint marches."""

    @staticmethod
    def forward(ctx, c, signal, problem: Problem):
        sim = problem.sim
        mat = speed_materials(sim, c.detach())
        source = Source(problem.source_position, signal.detach())
        # the forward traces; the adjoint pass recomputes or stores what it needs
        _, traces = simulate(sim, source, None, problem.sensors, _mat=mat)
        ctx.problem = problem
        ctx.save_for_backward(c, signal)
        return traces

    @staticmethod
    def backward(ctx, grad_traces):
        c, signal = ctx.saved_tensors
        problem = ctx.problem
        sim = problem.sim
        mat = speed_materials(sim, c.detach())
        source = Source(problem.source_position, signal.detach())
        dphi = grad_traces.contiguous()

        def objective(traces):
            return 0.0, dphi

        if problem.mode == "history":
            _, grads, _, info = sensitivity(sim, source, None, problem.sensors, objective,
                                            _mat=mat, _probe=True)
        else:
            _, grads, _, info = reconstruction_sensitivity(
                sim, source, None, problem.sensors, objective, strip_dtype=problem.strip_dtype,
                checkpoints=problem.checkpoints, _mat=mat, _probe=True,
            )
        cd = c.detach().to(sim.dtype)
        grad_c = grads["mass"] * (-2.0 / (cd * cd * cd))
        grad_c = torch.where(torch.isfinite(grad_c), grad_c, torch.zeros_like(grad_c))
        grad_signal = info["source"].to(signal.dtype)
        return grad_c.to(c.dtype), grad_signal, None


def wave_traces(c: torch.Tensor, signal: torch.Tensor, problem: Problem) -> torch.Tensor:
    """Differentiable receiver traces (N, num_sensors) of speed `c` and source `signal`."""
    as_position(problem.sim, problem.source_position)
    return WaveTraces.apply(c, signal, problem)
