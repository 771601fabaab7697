"""Scene sharding across ranks (one process per GPU).

Independent scenes need no exchange during a step, so a batch is split into
contiguous scene ranges, one per rank, balanced by body count; the only
collectives are the timing and work reductions after the timed region.
"""
from __future__ import annotations

import numpy as np


def scene_shards(scene_body_offset, world: int) -> list[tuple[int, int]]:
    """Contiguous scene ranges [s0, s1) per rank with about equal bodies."""
    off = np.asarray(scene_body_offset, dtype=np.int64)
    ns = len(off) - 1
    total = off[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        s = int(np.searchsorted(off, target, side="left"))
        s = min(max(s, bounds[-1]), ns)
        bounds.append(s)
    bounds.append(ns)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def reduce_timing(ms: float, work: float, device=None):
    """Max of the per-rank times and sum of the per-rank work."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    wk = torch.tensor([work], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(wk, op=dist.ReduceOp.SUM)
    return float(t.item()), float(wk.item())
