"""The multi-rank path of bench.py on CPU (gloo, world size 2): every rank
evaluates its own molecule (seed = rank), the job time is the slowest rank's
and the integral count the sum over ranks."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "pysisyphus-addons_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench

        t, n = bench.aggregate_over_ranks(dist, torch, 1.0 + rank, 1000 * (rank + 1), "cpu")
        from pysisyphus_addons.common.synthetic import config_workload

        coords = config_workload("cfg1", seed=rank).mol.coords
        out[rank] = (t, n, float(coords.sum()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_bench():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0][:2] == out[1][:2] == (2.0, 3000.0)
    # the ranks evaluated different molecules
    assert out[0][2] != out[1][2]
