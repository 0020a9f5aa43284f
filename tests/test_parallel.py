"""Realization sharding and the benchmark's cross-rank reductions on CPU
(gloo, two ranks): every realization lands on exactly one rank in the
reference's block order, and the reductions give max time / summed work."""
import os
import socket

import pytest

from hipft_b200.parallel import reduce_timing, split_realizations


@pytest.mark.parametrize("nr,world", [(64, 1), (64, 2), (64, 8), (5, 2), (5, 4), (7, 3), (1, 1)])
def test_split_covers_all_realizations_in_order(nr, world):
    seen = []
    for r in range(world):
        first, cnt = split_realizations(nr, world, r)
        seen.extend(range(first, first + cnt))
        assert cnt in (nr // world, nr // world + 1)
        if r < nr % world:
            assert cnt == nr // world + 1  # remainder to the low ranks (src/hipft.f90:1040-1043)
    assert seen == list(range(nr))


def test_split_rejects_bad_rank():
    with pytest.raises(ValueError):
        split_realizations(4, 2, 2)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        first, cnt = split_realizations(10, world, rank)
        got = [None] * world
        dist.all_gather_object(got, (first, cnt))
        t, w = reduce_timing(dist, "cpu", 100.0 + rank, float(cnt))
        q.put((rank, got, t, w))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharding_and_reductions():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, t, w in res:
        assert got == [(0, 5), (5, 5)]
        assert t == 101.0 and w == 10.0
