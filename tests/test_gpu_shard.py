"""Sharded enumeration through the library: two gloo ranks (processes), each
running its shard of the roots with the CUDA kernels on cuda:0, counts summed
by the all-reduce.  The ranks' kernels never wait on one another (the only
exchange is the CPU all-reduce after each rank's run)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import g2aimd
        from g2aimd.context import Context, Plan
        from g2aimd.shard import match_sharded, mce_sharded
        g = g2aimd.Graph.rmat(12, 16, seed=4).degeneracy_recoded()
        deg = g.degrees().astype(np.float64)
        with Context(0) as ctx:
            ctx.load(g)
            c, h = mce_sharded(ctx, world, rank, cost=deg * deg, hist_len=64, schedule="heuristic")
            m = match_sharded(ctx, Plan.preset(24), world, rank)
        q.put((rank, c, h.tolist(), m))
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_one_graph(g2, orc):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    from g2aimd.context import Plan
    g = g2.Graph.rmat(12, 16, seed=4).degeneracy_recoded()
    want = orc.mce(g, threads=8, hist_len=64)
    wm = orc.match(g, Plan.preset(24), threads=8)["count"]
    for rank, c, h, m in res:
        assert c == want["count"], rank
        assert np.array_equal(np.array(h, np.uint64), want["hist"]), rank
        assert m == wm, rank
