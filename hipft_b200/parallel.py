"""Realization sharding across ranks (one process per GPU).

HipFT's only parallel decomposition is over realizations: each MPI rank takes a
contiguous block, the remainder going to the low ranks
(set_local_number_of_realizations, src/hipft.f90:1033-1050).  Realizations
never exchange data, so a multi-GPU run is N independent shards; the only
collectives are the per-step timing and throughput reductions of the
benchmark (max of elapsed time, sum of work), done on the host group.
"""
from __future__ import annotations


def split_realizations(nr: int, world: int, rank: int):
    """(first index, count) of rank's block of nr realizations."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, rem = divmod(nr, world)
    cnt = base + (1 if rank < rem else 0)
    first = rank * base + min(rank, rem)
    return first, cnt


def reduce_timing(dist, device, elapsed_ms: float, work: float):
    """Max elapsed time and summed work over the process group."""
    import torch
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    w = torch.tensor([work], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())
