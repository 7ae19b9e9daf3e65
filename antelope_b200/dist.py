"""Multi-GPU plumbing: one process per GPU.

Two ways to use several GPUs.  Independent solves (scans, serving) need no
exchange: the list of solves is split across ranks in contiguous blocks (the
same split as the reference's ParaRange over k-points, utility.h:104-115) and
only timings are aggregated (the whole-job time is the maximum over ranks).
One large solve is split over k (`solve_sharded`): each rank propagates its
ParaRange block of the k-grid, the per-step k-sums are added with one
all-reduce (the reference's MPI_Reduce, antelope.cpp:482-512), and the output
arrays are assembled from the sum.
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


def solve_sharded(problem, precision: str | None = None, group=None, device=None, **opts):
    """One solve split over the ranks of `group` (default: the default process
    group; without torch.distributed, a single rank): rank r runs k-points
    para_range(Ntotal, world, r), the (Nt + 1) x width sums are all-reduced
    (sum, FP64) and every rank assembles the same outputs."""
    import torch.distributed as dist

    from .api import Solver

    on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if on else 1
    rank = dist.get_rank(group) if on else 0
    kb, ke = para_range(problem.dims.ntotal, world, rank)
    if precision is not None:
        opts["precision"] = precision
    s = Solver(problem, k_slice=(kb, ke), **opts)
    s.run()
    sums = s.sums()
    s.close()
    return reduce_and_assemble(problem, sums, group=group, device=device)


def reduce_and_assemble(problem, sums, group=None, device=None):
    """Add the ranks' (Nt + 1) x width k-sums (all-reduce, FP64) and assemble
    the output arrays from the total on every rank."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from .api import assemble

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        t = torch.from_numpy(np.ascontiguousarray(sums, dtype=np.float64)).to(device if device is not None else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        sums = t.cpu().numpy()
    return assemble(problem, np.ascontiguousarray(sums))
