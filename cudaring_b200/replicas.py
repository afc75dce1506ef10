"""Multi-GPU layout: independent replicas and batches sharded by system.

The reference runs one model per process on one GPU and has no data-path
exchange; a single system of the benchmark sizes does not shard without a
per-step halo exchange.  So N GPUs run N independent replicas (weak scaling),
and a batch of independent systems is split into contiguous blocks of
systems, one block per rank, with no collective on the data path.  The only
collectives are host-side: the device time of the slowest rank, and the
per-system results gathered in system order.

Every rank makes the same collective calls in the same order.  The helpers
work with the ``nccl`` backend on GPUs and with ``gloo`` on CPU (tests).
"""
from __future__ import annotations

import numpy as np


def shard_systems(sizes, world: int, rank: int) -> range:
    """The contiguous block of systems of ``rank``: boundaries placed where the
    running vertex count crosses k / world of the total, so blocks carry
    nearly equal work; every system belongs to exactly one rank."""
    sizes = np.asarray(sizes, dtype=np.int64)
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world size or rank")
    n = len(sizes)
    if n == 0:
        return range(0, 0)
    cum = np.cumsum(sizes)
    total = int(cum[-1])
    cuts = [0]
    for k in range(1, world):
        # first system whose running count reaches k/world of the total
        cuts.append(int(np.searchsorted(cum, total * k / world, side="left")) + 1)
    cuts.append(n)
    cuts = np.minimum(np.maximum.accumulate(np.asarray(cuts)), n)
    return range(int(cuts[rank]), int(cuts[rank + 1]))


def _device():
    import torch
    import torch.distributed as dist

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x: float, world: int) -> float:
    """The largest x over the ranks (the job's device time is the slowest rank's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    """x summed over the ranks (units processed by the whole job)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_per_system(local: list, world: int) -> list:
    """Per-system results of every rank's block, concatenated in system order
    (blocks are contiguous and ordered by rank)."""
    if world == 1:
        return list(local)
    import torch.distributed as dist

    parts = [None] * world
    dist.all_gather_object(parts, list(local))
    out = []
    for p in parts:
        out.extend(p)
    return out
