"""Ropes over several GPUs: one process per GPU, each stepping its own shard of ropes.

The substep shards with no collective on the data path: ropes interact only inside a rope-rope
contact group (`set_rope_contact(..., group_ropes=G)`: G consecutive ropes), meshes carry
per-env poses and read-only lattices, so whole contact groups go to one rank and every rank
builds its own RopeBatch from its shard. The one exchange is for differentiable runs whose
parameters are shared by ropes on several ranks (a material fitted across the batch): the
gradient of such a parameter is the sum of the ranks' partial gradients, one all-reduce of a
few floats per step (NCCL between GPUs, gloo on the CPU).

    import ropesim.sharding as sh
    mine = sh.shard_ropes(rope_verts, world, rank, group_ropes=G)   # rope indices of this rank
    b = ropesim.RopeBatch.from_ropes([ropes[r] for r in mine], ...)
    ...
    loss.backward()
    sh.allreduce_gradients([theta])                                  # theta.grad summed over ranks
"""
from __future__ import annotations

import numpy as np

__all__ = ["contact_groups", "shard_ropes", "shard_table", "allreduce_gradients"]


def contact_groups(num_ropes: int, group_ropes: int = 1):
    """The contact groups of a batch as (first rope, end rope) ranges: `group_ropes` consecutive
    ropes each (the last may be shorter), as RopeBatch.set_rope_contact forms them."""
    if num_ropes < 0 or group_ropes < 1:
        raise ValueError("num_ropes must be >= 0 and group_ropes >= 1")
    return [(g, min(num_ropes, g + group_ropes)) for g in range(0, num_ropes, group_ropes)]


def shard_table(rope_verts, world: int, group_ropes: int = 1):
    """Rank of every rope: whole contact groups, balanced by vertex count (longest-processing-time
    first: groups by decreasing vertex count, each to the rank with the fewest vertices so far,
    ties to the lower rank). A pure function of its arguments, so every rank computes the same
    table without communicating."""
    verts = np.asarray(rope_verts, np.int64).reshape(-1)
    if world < 1:
        raise ValueError("world must be >= 1")
    if (verts < 2).any():
        raise ValueError("every rope needs at least 2 vertices")
    groups = contact_groups(len(verts), group_ropes)
    size = np.array([int(verts[a:b].sum()) for a, b in groups], np.int64)
    order = sorted(range(len(groups)), key=lambda g: (-size[g], g))
    load = np.zeros(world, np.int64)
    table = np.empty(len(verts), np.int64)
    for g in order:
        r = int(np.argmin(load))
        load[r] += size[g]
        a, b = groups[g]
        table[a:b] = r
    return table


def shard_ropes(rope_verts, world: int, rank: int, group_ropes: int = 1):
    """Indices (ascending, so contact groups keep their caller order) of the ropes of `rank`."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    return np.nonzero(shard_table(rope_verts, world, group_ropes) == rank)[0]


def allreduce_gradients(params, group=None):
    """Sum the `.grad` of shared parameters over all ranks, in place, in one flat bucket (one
    collective per call whatever the number of tensors). Parameters without a gradient count as
    zero. Every rank must call it with the same parameters in the same order."""
    import torch
    import torch.distributed as dist

    params = list(params)
    if not params or not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return params
    grads = [p.grad if p.grad is not None else torch.zeros_like(p) for p in params]
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for p, g in zip(params, grads):
        n = g.numel()
        p.grad = flat[off:off + n].view_as(g).clone()
        off += n
    return params
