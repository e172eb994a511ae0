"""Many 2D problems stepped together: `simulate_batch`.

Shots of one design, or designs of uneven size and order (a topology optimisation's
population), each a `simulate` of its own, run as one native batch (cwb_batch_*): every
time step of every problem is one launch per stencil radius plus one launch for all the
receivers, chunks of steps replayed as a CUDA graph, the launches' thread count chosen by
timing a few steps (`tune`). Each problem keeps its own grid, order, time step, faces,
pml, damping, sources and receivers, and its own step count: a shorter run rests while
the longer ones finish. The results are those of `simulate` on each problem, bit for bit.

The reference runs one problem at a time (its `measure` / `misfit_gradient` loop over
shots, cuwave utils.py:369-459, spreading them over GPUs at most); this is the batched
form of that loop's forward passes.
"""

from __future__ import annotations

from collections.abc import Sequence

import torch

from . import _native as nat
from .wave import (
    Simulation,
    Source,
    as_position,
    device,
    flatten_indices,
    forward_ops,
    pml_memory,
    prepare_shot,
    require_off_held_walls,
    require_stepped,
)


def simulate_batch(sims: Sequence[Simulation], sources: Sequence[Source], indicators,
                   sensors=None, *, tune: bool = True) -> list:
    """`simulate(sims[i], sources[i], indicators[i], sensors[i])` for every i, stepped
    together.

    Every problem is 2D, float32, of a uniform stiffness (a speed model enters through
    1/m) and unmasked, with its sources on interior nodes (at most 32 of them).

    Returns a list of (field, traces) per problem, or the field alone where its sensors
    are None, as `simulate` returns them.
    """
    n = len(sims)
    if not (len(sources) == len(indicators) == n):
        raise ValueError("one source and one indicator per simulation")
    sensors = [None] * n if sensors is None else list(sensors)
    if len(sensors) != n:
        raise ValueError("one sensor set (or None) per simulation")
    dev = device()
    keep, items, results = [], [], []
    for sim, source, indicator, sens in zip(sims, sources, indicators, sensors):
        if sim.ndim != 2 or sim.precision != "float32" or sim.masked:
            raise NotImplementedError("a batch steps unmasked 2D float32 problems")
        mat = sim.build_materials(indicator)
        if not mat["uniform"]:
            raise NotImplementedError("a batch steps a uniform stiffness (speed through 1/m)")
        shot = prepare_shot(sim, mat, source.position, source.signal)
        require_off_held_walls(sim, shot.position)
        require_stepped(sim, shot.position, "source")
        if not shot.foldable or shot.lin.numel() > 32:
            raise NotImplementedError("a batch folds at most 32 sources, on interior nodes")
        if shot.signal.shape[0] < sim.N:
            raise ValueError(f"the signal has {shot.signal.shape[0]} rows for {sim.N} steps")
        U = torch.zeros((2, *sim.Nx_padded), dtype=sim.dtype, device=dev)
        memory = pml_memory(sim, 3, dev)
        a = nat.level(U, add=0, period=2)
        ops = forward_ops(sim, mat, a, nat.level(U, add=1, period=2), a, shot, memory)
        step = ops[0]
        record, um = nat.points(None, None), None
        if sens is not None:
            lin = flatten_indices(sim, as_position(sim, sens))
            um = torch.zeros((sim.N, lin.numel()), dtype=sim.dtype, device=dev)
            record = nat.points(lin, um)
            keep.append(lin)
        items.append(nat.BatchItem(sim.plan().handle.value, step, record, int(sim.N)))
        keep.extend([mat, shot, U, memory])
        results.append((sim, U, um))
    batch = nat.Batch(items)
    if tune:
        batch.tune(min(8, max(sim.N for sim in sims)))
    batch.march(0, max(sim.N for sim in sims))
    out = []
    for sim, U, um in results:
        field = U[(sim.N - 1) % 2][tuple(slice(0, k) for k in sim.Nx)]
        out.append(field if um is None else (field, um))
    torch.cuda.current_stream().synchronize()
    del batch, keep
    return out
