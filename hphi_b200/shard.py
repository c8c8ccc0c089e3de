"""Instance sharding across GPUs for the batched and served Lanczos modes.

Independent Hamiltonians need no exchange during a solve, so N GPUs (one process per GPU,
torch.distributed for the plumbing) split the instances and run their batches alone; the
only collectives are the final gather of the results and the max-over-ranks timing.  The
split balances the work (proportional to the sector dimension) greedily, largest first.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


def partition(dims: Sequence[int], world: int) -> List[List[int]]:
    """Instance indices for each rank: largest dimension first to the least-loaded rank.
    Every index appears on exactly one rank; each rank's list is in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(dims)), key=lambda k: (-int(dims[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += int(dims[i])
    return [sorted(p) for p in parts]


def gather(values: np.ndarray, indices: Sequence[int], n: int, dist=None) -> np.ndarray:
    """Assembles per-instance rows computed on each rank (values[k] belongs to instance
    indices[k]) into one (n, ...) array on every rank, in instance order."""
    values = np.asarray(values, dtype=np.float64)
    width = values.shape[1:] if values.ndim > 1 else ()
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        out = np.zeros((n,) + width)
        out[list(indices)] = values
        return out
    import torch
    world = dist.get_world_size()
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    flat = int(np.prod(width)) if width else 1
    # fixed-size exchange: every rank sends an (n, 1 + flat) buffer with a valid flag
    buf = torch.zeros((n, 1 + flat), dtype=torch.float64, device=dev)
    if len(indices):
        buf[list(indices), 0] = 1.0
        buf[list(indices), 1:] = torch.as_tensor(values.reshape(len(indices), flat), dtype=torch.float64, device=dev)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = np.zeros((n, flat))
    seen = np.zeros(n)
    for p in parts:
        p = p.cpu().numpy()
        m = p[:, 0] > 0.5
        out[m] = p[m, 1:]
        seen += m
    if not np.all(seen == 1):
        raise RuntimeError("shard.gather: every instance must come from exactly one rank")
    return out.reshape((n,) + width)


def max_over_ranks(t: float, dist=None) -> float:
    """The largest of the ranks' times (the job time of independent replicas)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(t)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    x = torch.tensor([float(t)], dtype=torch.float64, device=dev)
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    return float(x.item())
