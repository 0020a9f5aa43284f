"""Realization sharding across ranks (one process per GPU).

HipFT's only parallel decomposition is over realizations: each MPI rank takes a
contiguous block, the remainder going to the low ranks
(set_local_number_of_realizations, src/hipft.f90:1033-1050).  Realizations
never exchange field data.  Two ways to run them on several processes:

* replicas (the benchmark's weak scaling): every rank advances its block with
  its own time step; the only collectives are the benchmark's timing and
  throughput reductions;
* the reference's plain mode (``run_field_sharded``): one time step and one
  stage count for all realizations, kept by the four scalar MIN/MAX
  all-reduces the reference makes per step (src/hipft.f90:5036, 5103, 5141,
  7345), and the maps gathered on rank 0 for writing; the results are the same
  as one process holding every realization.
"""
from __future__ import annotations

import ctypes

import numpy as np


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


def run_field_sharded(namelist: str, run_dir: str, npm: int, ntm: int, n_realizations: int, device: int = 0):
    """This rank's part of a plain-mode run (hipft_run_shard) over the
    initialised torch.distributed group; returns its realizations' final
    field, shape (nr_local, npm, ntm).  All ranks share run_dir."""
    import torch
    import torch.distributed as dist
    from . import gpu
    rank, world = dist.get_rank(), dist.get_world_size()
    _, cnt = split_realizations(n_realizations, world, rank)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    errors = []

    def allreduce(user, op, value):
        try:
            t = torch.tensor([value[0]], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MIN if op == 0 else dist.ReduceOp.MAX)
            value[0] = float(t.item())
            return 0
        except Exception as e:  # reported through the library's status
            errors.append(e)
            return 1

    def gather(user, local, n_local, glob):
        try:
            mine = np.ctypeslib.as_array(local, shape=(int(n_local),)).copy()
            parts = [None] * world if rank == 0 else None
            dist.gather_object(mine, parts, dst=0)
            if rank == 0:
                allv = np.concatenate(parts)
                ctypes.memmove(glob, allv.ctypes.data, allv.nbytes)
            return 0
        except Exception as e:
            errors.append(e)
            return 1

    cb_red, cb_gat = gpu.ALLREDUCE_CB(allreduce), gpu.GATHER_CB(gather)
    sh = gpu.Shard(rank, world, cb_red, cb_gat, None)
    f = np.zeros((cnt, npm, ntm))
    rc = gpu.lib().hipft_run_shard(namelist.encode(), run_dir.encode(), int(device), ctypes.byref(sh),
                                   f.ctypes.data_as(gpu.DPTR), f.size)
    if rc:
        raise gpu.HipftError(rc, "hipft_run_shard", f"{namelist} {errors}")
    return f
