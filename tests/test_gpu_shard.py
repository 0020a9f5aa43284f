"""Plain-mode sharding: realizations split over two processes.

Two ranks (gloo on the host, both on one GPU; no kernel of one rank waits on
the other: the ranks exchange only host scalars and the gathered maps) run
hipft_run_shard on a 3-realization case (2 + 1, the reference's split,
src/hipft.f90:1025-1037) with differing diffusion coefficients, flows, PTL
subcycling and map output.  The four scalar all-reduces keep one time step,
so the result must equal the single-process run bit for bit: final fields,
every history file and every map file.
"""
import filecmp
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

import test_gpu_features as F

pytestmark = pytest.mark.gpu

CASE = dict(F.BASE, n_realizations=3, advance_flow=True, flow_dr_model=1, flow_mf_model=1,
            advance_diffusion=True, diffusion_coef_constants=[100.0, 500.0, 900.0],
            flow_dr_coef_p2_values=[-250.0, -300.0, -200.0], validation_run=1, strang_splitting=True,
            output_map_time_cadence=2.0, output_single_precision=False, time_end=6.0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nl, run_dir, out, npm, ntm, nr):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from hipft_b200.parallel import run_field_sharded
        f = run_field_sharded(nl, run_dir, npm, ntm, nr)
        np.save(os.path.join(out, f"f{rank}.npy"), f)
    finally:
        dist.destroy_process_group()


def test_sharded_run_equals_single_process(tmp_path):
    import torch.multiprocessing as mp
    import hipft_b200 as H
    text = F._namelist(CASE)
    one, two = tmp_path / "one", tmp_path / "two"
    one.mkdir()
    two.mkdir()
    for d in (one, two):
        (d / "hipft.in").write_text(text)
    ntm, npm, nr = CASE["res_nt"], CASE["res_np"] + 1, CASE["n_realizations"]
    mp.spawn(_worker, args=(2, _free_port(), str(two / "hipft.in"), str(two), str(tmp_path), npm, ntm, nr),
             nprocs=2, join=True)
    f_shard = np.concatenate([np.load(tmp_path / "f0.npy"), np.load(tmp_path / "f1.npy")])
    f_one = H.run_field(str(one / "hipft.in"), str(one), (nr, npm, ntm))
    assert np.array_equal(f_shard, f_one)
    for i in range(1, nr + 1):
        for kind in ("sol", "num"):
            name = f"hipft_history_{kind}_r{i:06d}.out"
            assert filecmp.cmp(one / name, two / name, shallow=False), name
    maps = sorted(p.name for p in (one / "output_maps").iterdir())
    assert len(maps) >= 3
    for m in maps:
        assert filecmp.cmp(one / "output_maps" / m, two / "output_maps" / m, shallow=False), m
    for m in ("hipft_brmap_initial.h5", "hipft_brmap_final.h5", "hipft_brmap_initial_0.h5",
              "hipft_brmap_final_analytic.h5", "hipft_output_map_list.out"):
        assert filecmp.cmp(one / m, two / m, shallow=False), m
