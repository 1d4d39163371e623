"""Multi-GPU use of the engine: independent replicas, no data-path collective.

The SINGLE_GPU path does not shard (one graph, resident in one GPU's HBM); N
GPUs run N replicas, each answering its own share of the root queries.  The
only cross-rank steps are a barrier and the max-over-ranks of each rank's
device time, which give the job's wall time.
"""
from __future__ import annotations

from typing import List, Sequence


def shard(items: Sequence, rank: int, world: int) -> List:
    """Round-robin share of `items` for `rank` (rank r takes r, r+W, ...)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return list(items[rank::world])


def max_over_ranks(value: float, device=None) -> float:
    """All-reduce MAX of a per-rank scalar (a timing), on the default group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
