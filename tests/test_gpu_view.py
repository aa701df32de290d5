"""Out-of-core runs over view bins on the GPU (g2_view_mce / g2_view_match):
the CSR stays in host memory, host threads build each bin's view, the device
enumerates view after view with the next upload overlapping the current run.
Totals, histograms and per-bin counts equal the oracle over the whole graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vctx(g2):
    from g2aimd.context import Context
    c = Context(0)
    yield c
    c.close()


def per_bin_oracle_mce(orc, g, bin_of, nbins, hist_len=64):
    out = np.zeros(nbins, np.uint64)
    for b in range(nbins):
        src = np.flatnonzero(bin_of == b).astype(np.uint32)
        if src.size:
            out[b] = orc.mce(g, roots=src, hist_len=hist_len)["count"]
    return out


@pytest.mark.parametrize("nbins,producers", [(1, 1), (7, 1), (7, 3), (64, 4)])
def test_view_mce_equals_oracle(vctx, orc, c1_graph, nbins, producers):
    g = c1_graph
    want = orc.mce(g, hist_len=64)
    bin_of = np.random.default_rng(nbins).integers(0, nbins, g.n).astype(np.uint32)
    count, hist, per_bin, st = vctx.view_mce(g, bin_of, nbins=nbins, hist_len=64, producers=producers)
    assert count == want["count"]
    assert np.array_equal(hist, want["hist"])
    assert int(per_bin.sum()) == count
    assert np.array_equal(per_bin, per_bin_oracle_mce(orc, g, bin_of, nbins))
    assert 1 <= st["bins"] <= nbins and st["h2d_bytes"] > 0 and st["view_edges"] > 0


def test_view_mce_many_bins_rmat(vctx, orc, g2):
    g = g2.Graph.rmat(11, 8, seed=2).degeneracy_recoded()
    want = orc.mce(g, hist_len=64)
    nb, bin_of = g.view_bins(max_bytes=96 << 10, radius=1, row_radius=1, min_root_degree=1)
    assert nb > 4
    count, hist, per_bin, st = vctx.view_mce(g, bin_of, hist_len=64, producers=2)
    assert count == want["count"] and np.array_equal(hist, want["hist"])
    assert 4 < st["bins"] <= nb


def test_view_mce_schedules_and_no_graph_after(vctx, orc, c1_graph):
    g = c1_graph
    want = orc.mce(g, hist_len=64)["count"]
    bin_of = (np.arange(g.n) % 5).astype(np.uint32)
    c, _, _, _ = vctx.view_mce(g, bin_of, hist_len=64, schedule="heuristic")
    assert c == want
    # the view run released the context's graph: a run needs a load first
    with pytest.raises(Exception):
        vctx.mce(hist_len=64)
    vctx.load(g)
    assert vctx.mce(hist_len=64)[0] == want


def test_view_roots_subset(vctx, orc, c1_graph):
    g = c1_graph
    bin_of = np.full(g.n, 0xFFFFFFFF, np.uint32)  # only even roots, in 3 bins
    bin_of[::2] = (np.arange(0, g.n, 2) // 700).astype(np.uint32)
    src = np.arange(0, g.n, 2, dtype=np.uint32)
    want = orc.mce(g, roots=src, hist_len=64)
    count, hist, per_bin, _ = vctx.view_mce(g, bin_of, hist_len=64)
    assert count == want["count"] and np.array_equal(hist, want["hist"])


@pytest.mark.parametrize("q", [0, 1, 2, 24])
def test_view_match_equals_oracle(vctx, orc, g2, q):
    from g2aimd.context import Plan
    g = g2.Graph.rmat(11, 8, seed=4).degeneracy_recoded()
    plan = Plan.preset(q)
    want = orc.match(g, plan, threads=4)["count"]
    sh = plan.view_shape()
    for no_upper in sorted({True, not sh["upper"]}):
        kw = dict(sh, upper=sh["upper"] and not no_upper, forward=sh["forward"] and not no_upper)
        nb, bin_of = g.view_bins(max_bytes=(8 << 10) if kw["forward"] else (32 << 10), **kw)
        assert nb > 8
        count, per_bin, st = vctx.view_match(g, bin_of, plan, producers=3, no_upper=no_upper)
        assert count == want, (q, no_upper, count, want)
        assert int(per_bin.sum()) == count
        assert st["bins"] >= 1


def test_view_match_plan_walk_handoff(vctx, orc, g2):
    """4-cycles with frequent hand-offs inside each view."""
    from g2aimd.context import Plan
    g = g2.Graph.rmat(10, 12, seed=6).degeneracy_recoded()
    plan = Plan.preset(1)
    want = orc.match(g, plan, threads=4)["count"]
    bin_of = (np.arange(g.n) % 3).astype(np.uint32)
    count, _, _ = vctx.view_match(g, bin_of, plan, spill_kcycles=1)
    assert count == want


def test_view_rejects_scores(vctx, c1_graph):
    bin_of = np.zeros(c1_graph.n, np.uint32)
    with pytest.raises(Exception):
        vctx.view_mce(c1_graph, bin_of, schedule="scores", scores=np.ones(c1_graph.n, np.float32))


def test_view_runs_with_bounded_pinned_buffers(vctx, orc, c1_graph):
    """g2_view_opts.slots (-qs) bounds the pinned view buffers: two of them for
    four producers, then a second run on the same context with fewer buffers
    than the first (the buffers beyond a call's count are released), each equal
    to the run with the default count."""
    g = c1_graph
    bin_of = (np.arange(g.n) % 9).astype(np.uint32)
    c0, h0, pb0, _ = vctx.view_mce(g, bin_of, hist_len=64, producers=4)
    assert c0 == orc.mce(g, hist_len=64)["count"]
    for slots in (4, 2):
        c, h, pb, _ = vctx.view_mce(g, bin_of, hist_len=64, producers=4, slots=slots)
        assert c == c0 and np.array_equal(h, h0) and np.array_equal(pb, pb0)
    from g2aimd.context import Plan
    want = orc.match(g, Plan.preset(24))["count"]
    c, pb, _ = vctx.view_match(g, bin_of, Plan.preset(24), producers=4, slots=2)
    assert c == want
    vctx.load(g)


@pytest.mark.parametrize("nbins", [1, 7, 64])
def test_device_built_views_mce(vctx, orc, c1_graph, nbins):
    """Views built by the GPU from the mapped host CSR (G2_VIEW_DEVICE) give
    the host-built views' sizes and per-bin results, and the oracle's totals."""
    g = c1_graph
    want = orc.mce(g, hist_len=64)
    bin_of = np.random.default_rng(nbins + 100).integers(0, nbins, g.n).astype(np.uint32)
    c_h, h_h, pb_h, st_h = vctx.view_mce(g, bin_of, nbins=nbins, hist_len=64, producers=2)
    c_d, h_d, pb_d, st_d = vctx.view_mce(g, bin_of, nbins=nbins, hist_len=64, device=True)
    assert c_d == c_h == want["count"]
    assert np.array_equal(h_d, want["hist"]) and np.array_equal(pb_d, pb_h)
    assert (st_d["bins"], st_d["view_vertices"], st_d["view_edges"]) == \
        (st_h["bins"], st_h["view_vertices"], st_h["view_edges"])
    vctx.load(g)


@pytest.mark.parametrize("q", [0, 24, 25])
def test_device_built_views_cliques(vctx, orc, g2, q):
    from g2aimd.context import Plan
    g = g2.Graph.rmat(12, 16, seed=4).degeneracy_recoded()
    plan = Plan.preset(q)
    nb, bin_of = g.view_bins(max_bytes=64 << 10, **plan.view_shape())
    assert nb > 2
    want = orc.match(g, plan, threads=8)["count"]
    c_h, pb_h, st_h = vctx.view_match(g, bin_of, plan, producers=2)
    c_d, pb_d, st_d = vctx.view_match(g, bin_of, plan, device=True)
    assert c_d == c_h == want and np.array_equal(pb_d, pb_h)
    assert (st_d["view_vertices"], st_d["view_edges"]) == (st_h["view_vertices"], st_h["view_edges"])
    vctx.load(g)


def test_device_built_views_need_radius_one(vctx, g2):
    from g2aimd._lib import G2Error
    from g2aimd.context import Plan
    g = g2.Graph.rmat(10, 8, seed=5).degeneracy_recoded()
    with pytest.raises(G2Error):  # 4-cycles need radius-2 views: host-built only
        vctx.view_match(g, (np.arange(g.n) % 3).astype(np.uint32), Plan.preset(1), device=True)
    vctx.load(g)


@pytest.mark.parametrize("shape", [dict(), dict(upper=True), dict(upper=True, forward=True), dict(forward=True)])
def test_device_built_view_bytes_equal_host_build(vctx, g2, shape):
    """g2_view_materialize_device gives the host builder's view exactly: row
    pointers, columns, forward offsets, sources, global ids, max forward degree
    (R-MAT s13 with a hub-heavy and a light root set; minimum root degree 3)."""
    g = g2.Graph.rmat(13, 16, seed=6).degeneracy_recoded()
    rng = np.random.default_rng(3)
    for src in (np.arange(g.n - 600, g.n, dtype=np.uint32), np.sort(rng.choice(g.n, 900, replace=False))):
        src = src.astype(np.uint32)
        h, hs, hid = g.view(src, radius=1, row_radius=1, min_root_degree=3, **shape)
        d, ds, did = vctx.view_device(g, src, min_root_degree=3, **shape)
        assert np.array_equal(h.row_ptrs, d.row_ptrs) and np.array_equal(h.cols, d.cols)
        assert np.array_equal(h.fwd_offsets, d.fwd_offsets) and h.max_fwd == d.max_fwd
        assert np.array_equal(hs, ds) and np.array_equal(hid, did)
    vctx.load(g)


def test_device_built_view_csr_sharing_pages_with_other_arrays(vctx, g2):
    """The host CSR is registered by its exact byte ranges: a pageable array
    that starts on the page where the columns end and runs past it (here the
    sources, copied to the device while the CSR is mapped) still copies."""
    g = g2.Graph.rmat(12, 16, seed=7).degeneracy_recoded()
    src = np.arange(g.n - 700, g.n, dtype=np.uint32)
    n, m = g.n, g.m
    buf = np.zeros(8 * (n + 1) + 4 * m + 4 * src.size + 3 * 4096, np.uint8)
    base = (-buf.ctypes.data) % 4096 + 64
    rp_at = base
    ci_at = rp_at + 8 * (n + 1)
    src_at = ci_at + 4 * m  # the offsets within a page are fixed: base is 64 bytes past a page start
    rp = buf[rp_at:rp_at + 8 * (n + 1)].view(np.uint64)
    ci = buf[ci_at:ci_at + 4 * m].view(np.uint32)
    sv = buf[src_at:src_at + 4 * src.size].view(np.uint32)
    rp[:], ci[:], sv[:] = g.row_ptrs, g.cols, src
    # the sources start on the page of the columns' last byte, and end past it
    # (pages of absolute addresses)
    a = buf.ctypes.data
    assert (a + src_at) // 4096 == (a + ci_at + 4 * m - 1) // 4096 < (a + src_at + 4 * src.size - 1) // 4096
    gb = g2.Graph(rp, ci)
    assert gb.row_ptrs.ctypes.data == rp.ctypes.data and gb.cols.ctypes.data == ci.ctypes.data
    for shape in (dict(), dict(upper=True, forward=True)):
        h, hs, hid = g.view(src, radius=1, row_radius=1, min_root_degree=2, **shape)
        d, ds, did = vctx.view_device(gb, sv, min_root_degree=2, **shape)
        assert np.array_equal(h.row_ptrs, d.row_ptrs) and np.array_equal(h.cols, d.cols)
        assert np.array_equal(hs, ds) and np.array_equal(hid, did)
    vctx.load(g)

