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
    """Sum a count and an optional histogram (uint64 values) over the ranks of
    `group`.  Collectives have no uint64 sum, so every value travels as its low
    and high 32-bit halves in int64 lanes (exact for up to 2^31 ranks) and is
    put back together here; a total of 2^64 or more raises OverflowError."""
    import torch
    import torch.distributed as dist
    vals = np.concatenate([np.asarray([int(count)], dtype=np.uint64),
                           np.zeros(0, np.uint64) if hist is None else np.asarray(hist, dtype=np.uint64)])
    halves = np.concatenate([vals & np.uint64(0xFFFFFFFF), vals >> np.uint64(32)]).astype(np.int64)
    t = torch.from_numpy(halves)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t = t.cpu().numpy()
    k = vals.size
    tot = [(int(t[k + i]) << 32) + int(t[i]) for i in range(k)]
    if any(x >= 1 << 64 for x in tot):
        raise OverflowError("a summed count does not fit in 64 bits")
    return tot[0], (None if hist is None else np.asarray(tot[1:], dtype=np.uint64))


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


NO_BIN = 0xFFFFFFFF


def shard_bins(bin_of, nbins: int, world: int, rank: int, cost=None):
    """This rank's part of a view-bin partition (the out-of-core path over
    several GPUs; the reference deals bins to `-cn` consumers through a shared
    queue, system/worker.h:214-262).  Bins go round robin, or longest first to
    the least-loaded rank when a per-bin cost is given (e.g. view bytes).
    Returns (local bin_of with other ranks' roots set to NO_BIN and this rank's
    bins renumbered 0..k-1, k, the global id of each local bin)."""
    mine = shard(nbins, world, rank, cost)
    local = np.full(nbins + 1, NO_BIN, dtype=np.uint32)
    local[mine] = np.arange(mine.size, dtype=np.uint32)
    b = np.asarray(bin_of, dtype=np.uint32)
    idx = np.where(b == NO_BIN, nbins, np.minimum(b, nbins)).astype(np.int64)
    if np.any((b != NO_BIN) & (b >= nbins)):
        raise ValueError("bin id out of range")
    return local[idx], int(mine.size), mine


def view_sharded(run, bin_of, nbins: int, world: int, rank: int, hist_len: int = 0, cost=None, device=None,
                 group=None):
    """Out-of-core enumeration over all ranks: run(local_bin_of, k) enumerates
    this rank's k bins (Context.view_mce / view_match on this rank's GPU) and
    returns (count, hist or None, per-bin counts); one all-reduce gives the
    totals: (count, hist or None, per-bin counts of all nbins bins)."""
    import torch
    import torch.distributed as dist
    local, k, ids = shard_bins(bin_of, nbins, world, rank, cost)
    if k:
        count, hist, per_bin = run(local, k)
    else:
        count, hist, per_bin = 0, (np.zeros(hist_len, np.uint64) if hist_len else None), np.zeros(0, np.uint64)
    h = np.zeros(hist_len, np.int64) if not hist_len else np.asarray(hist, dtype=np.int64)
    pb = np.zeros(nbins, np.int64)
    pb[ids] = np.asarray(per_bin, dtype=np.int64)[:k]
    t = torch.from_numpy(np.concatenate([[int(count)], h, pb]).astype(np.int64))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t = t.cpu().numpy()
    return (int(t[0]), (t[1:1 + hist_len].astype(np.uint64) if hist_len else None),
            t[1 + hist_len:].astype(np.uint64))


def view_mce_sharded(ctx, graph, bin_of, nbins: int, world: int, rank: int, hist_len: int = 256, cost=None,
                     device=None, group=None, **kw):
    """Maximal cliques of a host graph, view bins spread over the ranks."""
    def run(local, k):
        c, h, pb, _st = ctx.view_mce(graph, local, nbins=k, hist_len=hist_len, **kw)
        return c, h, pb
    return view_sharded(run, bin_of, nbins, world, rank, hist_len, cost, device, group)


def view_match_sharded(ctx, graph, plan, bin_of, nbins: int, world: int, rank: int, cost=None, device=None,
                       group=None, **kw):
    """Matches of `plan` in a host graph, view bins spread over the ranks."""
    def run(local, k):
        c, pb, _st = ctx.view_match(graph, local, plan, nbins=k, **kw)
        return c, None, pb
    return view_sharded(run, bin_of, nbins, world, rank, 0, cost, device, group)
