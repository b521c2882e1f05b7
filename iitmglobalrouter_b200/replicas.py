"""Independent replicas across ranks.

The routing path does not shard: batches run in sequence through one cost
state (every commit changes the costs the next batch reads) and a batch's
Fenwick tracks span the whole grid. So N processes, one per GPU, each route
their own copy of a design; nothing crosses between them on the data path.
Only the bookkeeping is collective: the step time is the maximum over ranks,
the whole-job rate counts every rank's nets, and a digest of each rank's
routed result checks that the replicas agree (routing is deterministic).
Every rank makes the same collective calls in the same order.
"""
from __future__ import annotations

import zlib

import numpy as np


def _world(dist) -> int:
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return 1
    return dist.get_world_size()


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of `value` over all ranks (the value itself on one rank)."""
    if _world(dist) == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, seconds: float, world: int) -> float:
    """Units per second of the whole job: every rank processed units_per_rank
    in at most `seconds` (the max over ranks)."""
    if seconds <= 0:
        raise ValueError("seconds must be positive")
    return world * units_per_rank / seconds


def digest(*arrays) -> int:
    """CRC-32 over the bytes of the given arrays, in order."""
    c = 0
    for a in arrays:
        c = zlib.crc32(np.ascontiguousarray(a).tobytes(), c)
    return c


def replicas_agree(d: int, dist=None, device=None) -> bool:
    """True when every rank passed the same digest."""
    if _world(dist) == 1:
        return True
    import torch

    t = torch.tensor([int(d)], dtype=torch.int64, device=device)
    lo = t.clone()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(lo, op=dist.ReduceOp.MIN)
    return int(t.item()) == int(lo.item())
