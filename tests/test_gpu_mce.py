"""Maximal clique enumeration on the GPU against the CPU oracle (bit-exact
count, size histogram and per-root search-tree size)."""
import numpy as np
import pytest

from helpers import random_graph, small_graphs

pytestmark = pytest.mark.gpu


def _same(got, want, name):
    c, h = got[0], got[1]
    assert c == want["count"], name
    assert np.array_equal(h[: want["hist"].size], want["hist"][: h.size]), name


def test_small_graphs(g2, orc, ctx):
    for g in small_graphs(g2.Graph):
        for recode in (False, True):
            gg = g.degeneracy_recoded() if recode else g
            ctx.load(gg)
            want = orc.mce(gg, per_root=True)
            c, h, rn = ctx.mce(root_nodes=True)
            _same((c, h), want, gg.name)
            assert np.array_equal(rn, want["root_nodes"]), gg.name


def test_config1_er_planted(orc, ctx, c1_graph):
    """ER(2000, 0.01) + 5 x K12: count, histogram and tree shape."""
    ctx.load(c1_graph)
    want = orc.mce(c1_graph, threads=4, per_root=True)
    c, h, rn = ctx.mce(root_nodes=True)
    _same((c, h), want, "c1")
    assert h[12] >= 5
    assert np.array_equal(rn, want["root_nodes"])


def test_rmat_and_schedules(g2, orc, ctx):
    g = g2.Graph.rmat(12, 16, seed=11).degeneracy_recoded()
    ctx.load(g)
    want = orc.mce(g, threads=8, per_root=True)
    for sched in ("given", "heuristic"):
        c, h, rn = ctx.mce(root_nodes=True, schedule=sched)
        _same((c, h), want, sched)
        assert np.array_equal(rn, want["root_nodes"]), sched
    scores = np.random.default_rng(0).random(g.n).astype(np.float32)
    c, h = ctx.mce(schedule="scores", scores=scores)
    _same((c, h), want, "scores")


def test_sources_subset_and_order(g2, orc, ctx):
    g = random_graph(g2.Graph, 400, 0.05, 3, planted=[tuple(range(0, 200, 17))]).degeneracy_recoded()
    ctx.load(g)
    src = np.random.default_rng(1).permutation(g.n)[:150].astype(np.uint32)
    want = orc.mce(g, roots=src, per_root=True)
    c, h, rn = ctx.mce(sources=src, root_nodes=True)
    _same((c, h), want, "subset")
    assert np.array_equal(rn, want["root_nodes"])
    c2, h2, rn2 = ctx.mce(sources=src, root_nodes=True, schedule="heuristic")
    assert c2 == c and np.array_equal(h2, h) and np.array_equal(rn2, rn)


def test_deferral_passes_with_tiny_scratch(g2, orc):
    """A slab too small for the big roots sends them through the deferred
    passes (bigger slab per warp); results do not change."""
    from g2aimd.context import Context
    g = g2.Graph.rmat(12, 16, seed=5).degeneracy_recoded()
    want = orc.mce(g, threads=8)
    with Context(0, scratch_bytes=32 << 20) as c:
        c.load(g)
        got = c.mce()
    _same(got, want, "tiny-scratch")


def test_not_degeneracy_ordered(g2, orc, ctx):
    """Raw R-MAT ids (hubs early): large forward sets, wide rows."""
    g = g2.Graph.rmat(11, 8, seed=21)
    ctx.load(g)
    want = orc.mce(g, threads=8)
    _same(ctx.mce(), want, "raw-ids")


def test_histogram_too_short_is_an_error(g2, ctx):
    g = g2.Graph.from_edges(6, [(a, b) for a in range(6) for b in range(a + 1, 6)])
    ctx.load(g)
    with pytest.raises(g2.G2Error):
        ctx.mce(hist_len=4)


def test_device_work_model_matches_oracle(g2, orc, ctx, c1_graph):
    """The work model W counted on the device equals the oracle's."""
    for g in (c1_graph, g2.Graph.rmat(11, 16, seed=2).degeneracy_recoded()):
        ctx.load(g)
        w = np.zeros(1, np.uint64)
        c, h = ctx.mce(work_bytes=w)
        want = orc.mce(g, threads=8)
        assert c == want["count"]
        assert int(w[0]) == want["work"], g.name


def test_chung_lu_power_law(g2, orc, ctx):
    g = g2.Graph.chung_lu(1 << 15, 2.3, 16.0, seed=3).degeneracy_recoded()
    ctx.load(g)
    want = orc.mce(g, threads=8, per_root=True)
    c, h, rn = ctx.mce(root_nodes=True, schedule="heuristic")
    _same((c, h), want, g.name)
    assert np.array_equal(rn, want["root_nodes"])


def test_spilled_records_keep_results(g2, orc, ctx, c1_graph):
    """Long tasks hand their pending branches to later waves as records (here
    as early as possible: after 1000 SM cycles); count, histogram, per-root
    tree size and the work model W stay the oracle's, with and without
    spilling, and with a slab small enough to defer records."""
    from g2aimd.context import Context
    graphs = (c1_graph, g2.Graph.rmat(12, 16, seed=11).degeneracy_recoded(),
              g2.Graph.chung_lu(1 << 15, 2.3, 16.0, seed=3).degeneracy_recoded())
    for g in graphs:
        ctx.load(g)
        want = orc.mce(g, threads=8, per_root=True)
        for kw in ({"spill_kcycles": 1}, {"spill_kcycles": 1, "schedule": "heuristic"}, {"flags": 16}):
            c, h, rn = ctx.mce(root_nodes=True, **kw)
            _same((c, h), want, (g.name, kw))
            assert np.array_equal(rn, want["root_nodes"]), (g.name, kw)
            records, pool = ctx.spill_stats()
            if kw.get("flags") == 16:
                assert records == 0 and pool == 0
            else:
                assert records > 0 and pool > 0, (g.name, kw)
            w = np.zeros(1, np.uint64)
            ctx.mce(work_bytes=w, **kw)
            assert int(w[0]) == want["work"], (g.name, kw)
    g = graphs[1]
    want = orc.mce(g, threads=8, per_root=True)
    with Context(0, scratch_bytes=32 << 20) as c:
        c.load(g)
        got = c.mce(root_nodes=True, spill_kcycles=1)
        _same(got, want, "tiny-scratch-spill")
        assert np.array_equal(got[2], want["root_nodes"])


def test_host_spill_pass(g2, orc):
    """Raw R-MAT ids give roots whose rows and frames exceed a 256 KiB device
    scratch even for one warp; they run on the spill slab and the results stay
    the oracle's.  Without a spill slab the run reports the overflow."""
    from g2aimd.context import Context
    g = g2.Graph.rmat(11, 16, seed=21)
    want = orc.mce(g, threads=8, per_root=True)
    with Context(0, scratch_bytes=256 << 10) as c:
        c.load(g)
        got = c.mce(root_nodes=True, flags=16)
        bad = np.nonzero(got[2] != want["root_nodes"])[0]
        src = np.repeat(np.arange(g.n), np.diff(g.row_ptrs.astype(np.int64)))
        p = np.bincount(src[g.cols > src], minlength=g.n)
        assert bad.size == 0, [(int(v), int(p[v]), int(got[2][v]), int(want["root_nodes"][v])) for v in bad[:8]]
        _same(got, want, "host-spill")
        c.set_host_spill(0)
        with pytest.raises(g2.G2Error):
            c.mce(flags=16)


def test_stream_spill_and_status(g2, orc):
    """g2_mce_run_device enqueues the spill pass in stream order: with a 256 KiB
    scratch the device counters still equal the oracle's and g2_run_status
    reports 0; without a spill slab it reports the roots left out
    (G2_ERR_OVERFLOW)."""
    import torch
    from g2aimd.context import Context
    g = g2.Graph.rmat(11, 16, seed=21)
    want = orc.mce(g, threads=8, hist_len=256)
    dev = torch.device("cuda", 0)
    st = torch.cuda.Stream(dev)
    out = torch.zeros(257, dtype=torch.int64, device=dev)
    with Context(0, scratch_bytes=256 << 10) as c:
        c.load(g)
        c.mce_device(out.data_ptr(), 256, stream=st.cuda_stream, flags=16)
        assert c.run_status(st.cuda_stream) == 0
        h = out.cpu().numpy().astype(np.uint64)
        _same((int(h[0]), h[1:]), want, "stream spill")
        c.set_host_spill(0)
        c.mce_device(out.data_ptr(), 256, stream=st.cuda_stream, flags=16)
        assert c.run_status(st.cuda_stream) == -5  # G2_ERR_OVERFLOW
        assert int(out[0].item()) <= want["count"]
    with Context(0) as c:
        c.load(g)
        c.mce_device(out.data_ptr(), 256, stream=st.cuda_stream)
        assert c.run_status(st.cuda_stream) == 0 and int(out[0].item()) == want["count"]

