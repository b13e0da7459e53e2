"""Multi-GPU sharding of one probability over random shifts.

The Genz estimate is a mean over independent randomisations (shifts); each
shift's mean over the points is independent of every other shift given U, a
and b.  One process per GPU therefore owns a disjoint block of shifts, runs
the whole qmc_pnorm! pass on it with no data-path communication, and a
single all-gather of the per-shift means (n_reps doubles) produces the
estimate and its 3*SEM on every rank (src/qmc.jl:814-815).

Used by bench.py for --gpus N (weak scaling: every rank keeps the
single-GPU shift count) and covered on CPU by tests with the gloo backend.
"""
from __future__ import annotations

import math

import numpy as np


def shift_block(rank: int, world: int, n_reps_total: int) -> tuple[int, int]:
    """[start, stop) of the shifts owned by rank (contiguous, balanced)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n_reps_total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def combine(reps: np.ndarray) -> tuple[float, float]:
    """Mean over shifts and 3*SEM, exactly as qmc_pnorm! forms them."""
    n = reps.size
    total = 0.0
    for v in reps:  # in shift order, as sum(D.qmc_reps) over a short vector
        total += float(v)
    result = total / n
    acc = 0.0
    for v in reps:
        acc += (v - result) ** 2 / n
    return result, 3.0 * math.sqrt(acc / (n - 1))


def gather_reps(local_reps: np.ndarray, n_reps_total: int, group=None) -> np.ndarray:
    """All-gather the per-shift means of every rank into shift order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    counts = [shift_block(r, world, n_reps_total) for r in range(world)]
    width = max(b - a for a, b in counts)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    buf = torch.zeros(width, dtype=torch.float64, device=dev)
    buf[: local_reps.size] = torch.from_numpy(np.asarray(local_reps, dtype=np.float64)).to(dev)
    out = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    parts = [o[: b - a].cpu().numpy() for o, (a, b) in zip(out, counts)]
    return np.concatenate(parts)
