"""Root sharding over ranks (host logic of the multi-GPU path), checked with
world_size-2 gloo process groups on the CPU.  The oracle stands in for each
rank's device run; the shards, the cost balancing and the all-reduce of the
count and the clique-size histogram are the library's."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from g2aimd.shard import shard


def test_shards_partition_the_roots():
    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 1000):
        cost = rng.random(n) ** 4
        for world in (1, 2, 3, 8):
            for c in (None, cost):
                parts = [shard(n, world, r, c) for r in range(world)]
                allr = np.concatenate(parts) if parts else np.zeros(0)
                assert np.array_equal(np.sort(allr), np.arange(n)), (n, world)
                for p in parts:
                    assert np.all(np.diff(p.astype(np.int64)) > 0)


def test_cost_balanced_shards_are_balanced():
    rng = np.random.default_rng(1)
    cost = rng.pareto(1.5, 5000) + 0.01
    world = 4
    loads = [cost[shard(cost.size, world, r, cost)].sum() for r in range(world)]
    # LPT: every rank within the largest single cost of the mean
    assert max(loads) - min(loads) <= cost.max() + 1e-9
    rr = [cost[shard(cost.size, world, r)].sum() for r in range(world)]
    assert max(loads) <= max(rr) + 1e-9


def test_bad_rank_rejected():
    with pytest.raises(ValueError):
        shard(10, 2, 2)
    with pytest.raises(ValueError):
        shard(10, 2, 0, cost=np.ones(3))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import g2aimd
        import orc
        from g2aimd.context import Plan
        from g2aimd.shard import allreduce_counts
        g = g2aimd.Graph.er(300, 0.08, planted=2, planted_size=9, seed=5).degeneracy_recoded()
        deg = g.degrees().astype(np.float64)
        roots = shard(g.n, world, rank, cost=deg * deg)
        part = orc.mce(g, roots=roots, hist_len=32)
        c, h = allreduce_counts(part["count"], part["hist"])
        plan = Plan.preset(24)
        mc = orc.match(g, plan, roots=shard(g.n, world, rank))["count"]
        m, _ = allreduce_counts(mc)
        q.put((rank, c, h.tolist(), m))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_sharded_counts(g2, orc):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = g2.Graph.er(300, 0.08, planted=2, planted_size=9, seed=5).degeneracy_recoded()
    want = orc.mce(g, hist_len=32)
    from g2aimd.context import Plan
    wm = orc.match(g, Plan.preset(24))["count"]
    for rank, c, h, m in res:
        assert c == want["count"], rank
        assert np.array_equal(np.array(h, np.uint64), want["hist"]), rank
        assert m == wm, rank


def test_bin_shards_partition_the_bins():
    from g2aimd.shard import NO_BIN, shard_bins
    rng = np.random.default_rng(4)
    n, nbins = 500, 13
    bin_of = rng.integers(0, nbins, n).astype(np.uint32)
    bin_of[::17] = NO_BIN  # not roots
    for world in (1, 2, 3, 5):
        for cost in (None, rng.random(nbins)):
            seen = np.zeros(nbins, np.int64)
            for r in range(world):
                local, k, ids = shard_bins(bin_of, nbins, world, r, cost)
                assert ids.size == k
                seen[ids] += 1
                mine = local != NO_BIN
                # a root is this rank's exactly when its bin is, renumbered in order
                assert np.array_equal(mine, np.isin(bin_of, ids))
                assert np.array_equal(ids[local[mine]], bin_of[mine])
            assert np.all(seen == 1)
    with pytest.raises(ValueError):
        shard_bins(np.array([0, 5], np.uint32), 3, 1, 0)


def _view_rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import g2aimd
        import orc
        from g2aimd.context import Plan
        from g2aimd.shard import view_sharded
        g = g2aimd.Graph.er(300, 0.08, planted=2, planted_size=9, seed=5).degeneracy_recoded()
        nbins = 7
        bin_of = (np.arange(g.n) * 5 % nbins).astype(np.uint32)

        def oracle_over_views(shape, plan=None):
            # the oracle over each view stands in for this rank's device run
            def run(local, k):
                count, hist, per = 0, np.zeros(32, np.uint64), np.zeros(k, np.uint64)
                for b in range(k):
                    v, src, _ = g.view(np.flatnonzero(local == b).astype(np.uint32), **shape)
                    if not src.size:
                        continue
                    r = orc.mce(v, roots=src, hist_len=32) if plan is None else orc.match(v, plan, roots=src)
                    per[b] = r["count"]
                    count += r["count"]
                    if plan is None:
                        hist += r["hist"]
                return count, (hist if plan is None else None), per
            return run

        mce_shape = {"radius": 1, "row_radius": 1, "min_root_degree": 1}
        c, h, per = view_sharded(oracle_over_views(mce_shape), bin_of, nbins, world, rank, hist_len=32)
        plan = Plan.preset(24)
        m, _, mper = view_sharded(oracle_over_views(plan.view_shape(), plan), bin_of, nbins, world, rank,
                                  cost=np.arange(nbins, dtype=np.float64))
        q.put((rank, c, h.tolist(), per.tolist(), m, mper.tolist()))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_view_bins(g2, orc):
    """View bins dealt over two ranks: totals, histogram and per-bin counts."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_view_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = g2.Graph.er(300, 0.08, planted=2, planted_size=9, seed=5).degeneracy_recoded()
    from g2aimd.context import Plan
    want = orc.mce(g, hist_len=32)
    wm = orc.match(g, Plan.preset(24))["count"]
    nbins = 7
    bin_of = (np.arange(g.n) * 5 % nbins).astype(np.uint32)
    want_per = [orc.mce(g, roots=np.flatnonzero(bin_of == b).astype(np.uint32), hist_len=32)["count"]
                for b in range(nbins)]
    for rank, c, h, per, m, mper in res:
        assert c == want["count"] and np.array_equal(np.array(h, np.uint64), want["hist"]), rank
        assert per == want_per, rank
        assert m == wm and sum(mper) == wm, rank


def _lost_rank_main(rank, world, port, q):
    import datetime
    import time

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=4))
    from g2aimd.shard import allreduce_counts
    def report(msg):
        q.put((rank, msg))
        q.close()
        q.join_thread()  # the message is out before the process ends

    if rank == 1:
        report("left")  # this rank leaves between steps: no collective in flight
        os._exit(0)
    t0 = time.time()
    try:
        allreduce_counts(5, np.zeros(3, np.uint64))
        report("completed")
    except Exception as e:  # the survivor learns of it from the collective's timeout
        report(f"error after {time.time() - t0:.1f} s: {type(e).__name__}")
    os._exit(0)


def test_gloo_lost_rank_ends_in_an_error_not_a_hang():
    """A rank that leaves before the final all-reduce: the other rank's
    collective ends with an error within the process group's timeout."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_lost_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert res[1] == "left"
    assert res[0].startswith("error after"), res[0]
    assert float(res[0].split()[2]) < 60


def _big_rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from g2aimd.shard import allreduce_counts
        # totals at and above 2^63, where an int64 sum would wrap
        mine = (1 << 63) + 5 if rank == 0 else 1 << 62
        c, h = allreduce_counts(mine, np.array([(1 << 62) + rank, 7, 0], np.uint64))
        try:
            allreduce_counts((1 << 64) - 1)  # the sum needs 65 bits
            over = False
        except OverflowError:
            over = True
        q.put((rank, c, h.tolist(), over))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_allreduce_is_exact_for_uint64():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_big_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, c, h, over in res:
        assert c == (1 << 63) + (1 << 62) + 5, rank
        assert h == [(1 << 63) + 1, 14, 0], rank
        assert over, rank
