"""The multi-rank path on the CPU: two `gloo` ranks over 127.0.0.1.

The solver shards with no data-path collective: every rank steps its own whole contact groups
of ropes (ropesim.sharding), and the only collectives are the max over ranks of the timed totals
(bench.py) and, for differentiable runs, the sum over ranks of shared-parameter gradients
(ropesim.sharding.allreduce_gradients). With world size 2 on the CPU this checks that
  * the shard table gives every rope to exactly one rank, whole contact groups, balanced;
  * the ranks' shards, stepped independently (the FP64 oracle stands in for the GPU here),
    reproduce the single-process run to FP64 rounding (initial frames are transported along the
    flat rope array across rope boundaries, as in the reference, so a shard's first rope starts
    from a different predecessor's frame: last-bit differences, 1e-15 m here);
  * the all-reduced gradient of a parameter shared by every rope (a global EA multiplier, from
    the oracle adjoint of each shard) equals the single-process gradient;
  * bench.py's max over ranks and whole-job rate.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cosserat-rod-solver-cuda_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import ropesim.sharding as sh  # noqa: E402  (pure host code: no GPU needed)


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_table_whole_groups_balanced():
    rng = np.random.default_rng(0)
    verts = rng.integers(16, 257, 101)
    for world in (1, 2, 3, 8):
        for G in (1, 4):
            table = sh.shard_table(verts, world, G)
            assert table.shape == (101,) and table.min() >= 0 and table.max() < world
            for a, b in sh.contact_groups(101, G):
                assert (table[a:b] == table[a]).all()  # a contact group never straddles ranks
            shards = [sh.shard_ropes(verts, world, r, G) for r in range(world)]
            assert sorted(np.concatenate(shards).tolist()) == list(range(101))
            load = np.array([verts[s].sum() for s in shards])
            biggest = max(verts[a:b].sum() for a, b in sh.contact_groups(101, G))
            assert load.max() - load.min() <= biggest  # LPT: within one group of each other
    with pytest.raises(ValueError):
        sh.shard_ropes(verts, 2, 2)
    with pytest.raises(ValueError):
        sh.shard_table([5, 1], 2)


def _forward(ropes, sel):
    import ropesim_oracle as ro

    b = ro.RopeBatch.from_ropes([ropes[r] for r in sel], 0.117, 2000.0, 1e-3, 1 / 6000, 8)
    b.set_gravity((0.0, 0.0, -9.81))
    b.damping = 0.0
    b.drag = 0.2
    b.set_planes([[0.0, 0.0, 1.0, 0.0]], radius=0.005)
    for _ in range(3):
        b.step_free(1 / 60, 50)
    P = np.asarray(b.positions(), np.float64).reshape(-1, 3)
    out, o = {}, 0
    for r in sel:
        out[int(r)] = P[o:o + len(ropes[r])]
        o += len(ropes[r])
    return out


def _shared_ea_gradient(sel, R_total):
    """d(loss)/d(theta) at theta = 1 for EA_i = theta * EA0_i, where the loss is the global one
    (mean over all R_total ropes of the tip loss) restricted to the ropes `sel`."""
    import adjoint_cases as ac
    import ropesim_oracle as ro

    _, pos = ac.scene(R=R_total, V=12, plane=True, material="c1")
    seg, dens, ea0, ei0 = ac.MATERIALS["c1"]
    b = ro.RopeBatch.from_positions(pos[sel], dens, ea0, ei0, 1 / 6000, 8)
    b.set_gravity((0.0, 0.0, -9.81))
    b.damping = 0.0
    b.drag = 0.2
    b.set_planes([[0.0, 0.0, 1.0, 0.0]], radius=0.00635, mu_s=0.5, mu_k=0.3)
    progs = [p[:, sel] for p in ac.programs(pos, 2)]
    tgt = ac.targets(pos, 2)[:, sel]
    _, g = ac.oracle_loss_and_grad(b, progs, tgt, 1 / 60, 100, 12)
    ea = np.full(len(sel) * 12, ea0)
    return float((g["g_ea"] * ea).sum()) * len(sel) / R_total


def _rank_main(rank, world, port, out):
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import bench
    import scenarios as S

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        # bench.py's reduction: per-rank timed totals, rank 1 the slower one
        worst = bench.max_over_ranks(100.0 + 25.0 * rank, dist, "cpu")
        rate = bench.job_rate(world, 8 * 64 * 100, worst * 1e-3)
        # the forward: whole contact groups (G = 2) per rank, stepped by this rank alone
        ropes = S.uneven_ropes(7, 3, lo=16, hi=48)
        verts = [len(r) for r in ropes]
        mine = sh.shard_ropes(verts, world, rank, group_ropes=2)
        parts = [None] * world
        dist.all_gather_object(parts, _forward(ropes, mine))
        # the gradient of a parameter shared by every rope: partial on this rank's ropes, summed
        R = 6
        sel = sh.shard_ropes([12] * R, world, rank)
        theta = torch.ones(1, dtype=torch.float64, requires_grad=True)
        theta.grad = torch.tensor([_shared_ea_gradient(sel, R)], dtype=torch.float64)
        sh.allreduce_gradients([theta])
        out[rank] = (worst, rate, mine.tolist(), parts, float(theta.grad[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_and_gradient_allreduce():
    import torch.multiprocessing as mp

    import scenarios as S

    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0, f"rank exited with {p.exitcode}"
    res = dict(out)
    assert sorted(res) == [0, 1]
    ropes = S.uneven_ropes(7, 3, lo=16, hi=48)
    whole = _forward(ropes, np.arange(7))
    g_whole = _shared_ea_gradient(np.arange(6), 6)
    assert set(res[0][2]).isdisjoint(res[1][2]) and sorted(res[0][2] + res[1][2]) == list(range(7))
    for r in range(world):
        worst, rate, mine, parts, g = res[r]
        assert worst == pytest.approx(125.0)  # the slowest rank's total on every rank
        assert rate == pytest.approx(2 * 8 * 64 * 100 / 0.125)
        merged = {k: v for part in parts for k, v in part.items()}
        assert sorted(merged) == list(range(7))
        for k in range(7):  # the shards reproduce the single-process run to FP64 rounding
            np.testing.assert_allclose(merged[k], whole[k], rtol=0, atol=1e-12)
        assert g == pytest.approx(g_whole, rel=1e-12, abs=1e-300)
    assert abs(g_whole) > 0.0
