"""The multi-rank path of bench.py on the CPU: two `gloo` ranks over 127.0.0.1.

The solver shards with no data-path collective: every rank steps its own ropes (seeded by rank)
and the only collective is the max over ranks of the timed totals, from which the whole-job
rate is computed (weak scaling). This test runs that logic with world size 2 on the CPU:
max_over_ranks must return the slowest rank's time on every rank, the per-rank inputs must be
distinct shards, and the job rate must count both ranks' work over the slowest rank's time.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        # per-rank timed totals: rank 1 is the slower one
        ms = 100.0 + 25.0 * rank
        worst = bench.max_over_ranks(ms, dist, "cpu")
        pos, p0, v0, p1 = bench.c2_inputs(8, 2, 1234 + rank)
        shard = float(np.asarray(p1).sum())
        shards = [None] * world
        dist.all_gather_object(shards, shard)
        rate = bench.job_rate(world, 8 * 64 * 100, worst * 1e-3)
        out[rank] = (worst, shards, rate)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_and_sharding():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0, f"rank exited with {p.exitcode}"
    res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        worst, shards, rate = res[r]
        assert worst == pytest.approx(125.0)          # the slowest rank's total on every rank
        assert shards[0] != shards[1]                 # each rank steps its own ropes
        assert rate == pytest.approx(2 * 8 * 64 * 100 / 0.125)
