"""Root sharding over several GPUs (one process per GPU, torch.distributed).

Every maximal clique is found from exactly one root (its lowest vertex in the
id order) and every match from exactly one source, so the roots of one graph
split into disjoint shards with no exchange during enumeration: each rank runs
its shard on a replica of the CSR and one all-reduce of the counts (and the
clique-size histogram) ends the job.  This replaces the reference's bins over
`-cn` GPUs summed on the host (system/worker.h:214-279).

Shards are balanced by a per-root cost estimate when one is given (longest
processing time first: roots in descending cost, each to the least-loaded
rank), else dealt round-robin, which interleaves the heavy roots that a
degeneracy order puts at the end of the id range.
"""
from __future__ import annotations

import heapq

import numpy as np


def shard(n: int, world: int, rank: int, cost=None) -> np.ndarray:
    """Roots (uint32, ascending) of `rank` out of `world` for a graph of n vertices."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    if cost is None:
        return np.arange(rank, n, world, dtype=np.uint32)
    cost = np.asarray(cost, dtype=np.float64)
    if cost.shape != (n,):
        raise ValueError("cost must have one entry per vertex")
    order = np.lexsort((np.arange(n), -cost))  # descending cost, ties by id
    owner = np.empty(n, dtype=np.int64)
    heap = [(0.0, r) for r in range(world)]
    for v in order:
        load, r = heapq.heappop(heap)
        owner[v] = r
        heapq.heappush(heap, (load + float(cost[v]), r))
    return np.nonzero(owner == rank)[0].astype(np.uint32)


def allreduce_counts(count: int, hist=None, device=None, group=None):
    """Sum a count and an optional histogram over the ranks of `group`."""
    import torch
    import torch.distributed as dist
    h = np.zeros(0, np.int64) if hist is None else np.asarray(hist, dtype=np.int64)
    t = torch.from_numpy(np.concatenate([[int(count)], h]).astype(np.int64))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t = t.cpu().numpy()
    return int(t[0]), (None if hist is None else t[1:].astype(np.uint64))


def mce_sharded(ctx, world: int, rank: int, cost=None, hist_len: int = 256, device=None, group=None, **kw):
    """Maximal cliques of the graph loaded in `ctx`, this rank's shard on this
    rank's GPU, totals over all ranks: (count, hist)."""
    roots = shard(ctx.n, world, rank, cost)
    c, h = ctx.mce(sources=roots, hist_len=hist_len, **kw) if roots.size else (0, np.zeros(hist_len, np.uint64))
    return allreduce_counts(c, h, device=device, group=group)


def match_sharded(ctx, plan, world: int, rank: int, cost=None, device=None, group=None, **kw):
    """Matches of `plan` in the graph loaded in `ctx` over all ranks' shards."""
    roots = shard(ctx.n, world, rank, cost)
    c = ctx.match(plan, sources=roots, **kw) if roots.size else 0
    return allreduce_counts(c, None, device=device, group=group)[0]
