"""Multi-GPU plumbing: one process per GPU, independent solves per rank.

The propagation needs no exchange between solves, so a multi-GPU run
shards the list of solves across ranks (contiguous blocks, the same split as
the reference's ParaRange over k-points, utility.h:104-115) and only
aggregates timings: the whole-job time is the maximum over ranks.
"""
from __future__ import annotations


def para_range(total: int, size: int, rank: int) -> tuple[int, int]:
    """[start, end) of rank's block of `total` units (ParaRange)."""
    w1, w2 = divmod(total, size)
    start = w1 * rank + min(w2, rank)
    end = start + w1 + (1 if w2 > rank else 0)
    return start, end


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over the ranks of the default process group (the
    value itself when torch.distributed is not initialised)."""
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
