"""Instance sharding of the batched linear form across GPUs.

The instances of a batch (many initial conditions on one grid) are
independent, so with one process per GPU each rank takes a contiguous,
balanced range of them and steps it with no exchange at all; only the
outputs are gathered at the end (the gauge series), with one all_gather over
the process group: NCCL between GPUs, gloo on CPU.  Instance b always gets
the same initial condition whatever the number of ranks, so results do not
depend on the partition.
"""
from __future__ import annotations

import numpy as np


def instance_range(nbatch: int, world: int, rank: int):
    """(first, count) of the instances rank `rank` of `world` owns:
    contiguous, sizes differing by at most one, lower ranks first."""
    if nbatch < 0 or world < 1 or not (0 <= rank < world):
        raise ValueError("bad nbatch / world / rank")
    base, extra = divmod(nbatch, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def gather_instance_series(local: np.ndarray, nbatch: int, world: int, rank: int, group=None) -> np.ndarray:
    """All-gather per-rank series of shape (T, count, ...) along the instance
    axis into (T, nbatch, ...) in global instance order, on every rank."""
    import torch
    import torch.distributed as dist
    first, count = instance_range(nbatch, world, rank)
    local = np.asarray(local)
    if local.shape[1] != count:
        raise ValueError(f"rank {rank} holds {local.shape[1]} instances, expected {count}")
    cmax = -(-nbatch // world)
    shape = (local.shape[0], cmax) + local.shape[2:]
    pad = np.zeros(shape, dtype=np.float64)
    pad[:, :count] = local
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(pad).to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out = np.empty((local.shape[0], nbatch) + local.shape[2:], dtype=np.float64)
    for r, p in enumerate(parts):
        f, c = instance_range(nbatch, world, r)
        out[:, f:f + c] = p[:, :c].cpu().numpy()
    return out
