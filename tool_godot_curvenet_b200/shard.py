"""Sharding of a batch of independent meshes over ranks (one process per GPU).

Meshes are independent units, so the batch shards with no collective on the
data path: each rank builds and solves its own meshes; only timings and
statistics are reduced at the end.  The partition balances the estimated
cost (nnz of A plus the two triangular factors, a proxy for the bytes one
PCG iteration moves) with the longest-processing-time rule: meshes by
decreasing cost, each to the currently least-loaded rank.  Every rank
computes the same partition from the same inputs.
"""
import numpy as np


def mesh_cost(n_verts, n_tris):
    """Cost proxy of one mesh: about 7 entries per row of A and 3 per row of L."""
    return int(n_verts) * 13 + int(n_tris)


def lpt_partition(costs, world):
    """Indices of the meshes of each rank (lists, in increasing mesh order)."""
    costs = np.asarray(costs, dtype=np.int64)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world, dtype=np.int64)
    parts = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def rank_share(costs, world, rank):
    """The meshes of `rank` under the LPT partition (same on every rank)."""
    return lpt_partition(costs, world)[rank]


def reduce_over_ranks(dist, world, value, op="max", device="cpu"):
    """Reduce one host float over the ranks (identity with one rank).  Device
    timings are taken per rank with CUDA events; the job's time is their max.
    `device`: where the one-element tensor lives ("cuda:<local>" under NCCL,
    "cpu" under gloo)."""
    if world == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())
