"""Plan-driven subgraph counts on the GPU against the CPU oracle."""
import numpy as np
import pytest

from helpers import random_graph

pytestmark = pytest.mark.gpu

QUERIES = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 16, 17, 18, 23, 24, 25, 26]


@pytest.mark.parametrize("q", QUERIES)
def test_presets_small(g2, orc, ctx, q):
    from g2aimd.context import Plan
    plan = Plan.preset(q)
    k = plan.k
    for g in (random_graph(g2.Graph, 40 if k < 6 else 30, 0.3, 5 + q, planted=[tuple(range(0, 9))]),
              g2.Graph.rmat(9 if k < 6 else 8, 8, seed=q).degeneracy_recoded()):
        ctx.load(g)
        want = orc.match(g, plan)["count"]
        assert ctx.match(plan) == want, (q, g.name)
        assert ctx.match(plan, intersect_mode=1) == want, (q, g.name, "generic")


@pytest.mark.parametrize("q", [0, 1, 2, 24, 25])
def test_rmat_s13(g2, orc, ctx, q):
    from g2aimd.context import Plan
    g = g2.Graph.rmat(13, 16, seed=3).degeneracy_recoded()
    plan = Plan.preset(q)
    ctx.load(g)
    want = orc.match(g, plan, threads=8)["count"]
    assert ctx.match(plan) == want
    assert ctx.match(plan, schedule="heuristic") == want
    # the 40-register build of the kernel (6 CTAs of 256 threads per SM)
    assert ctx.match(plan, schedule="heuristic", ctas_per_sm=6) == want
    assert ctx.match(plan, ctas_per_sm=6, warps_per_block=4, intersect_mode=1) == want


def test_raw_ids_and_sources(g2, orc, ctx):
    from g2aimd.context import Plan
    g = g2.Graph.rmat(12, 8, seed=8)
    ctx.load(g)
    src = np.arange(0, g.n, 3, dtype=np.uint32)
    for q in (0, 2, 24):
        plan = Plan.preset(q)
        assert ctx.match(plan, sources=src) == orc.match(g, plan, roots=src, threads=8)["count"]


def test_empty_and_tiny(g2, ctx):
    from g2aimd.context import Plan
    ctx.load(g2.Graph.from_edges(5, []))
    assert ctx.match(Plan.preset(0)) == 0
    ctx.load(g2.Graph.from_edges(3, [(0, 1), (1, 2), (0, 2)]))
    assert ctx.match(Plan.preset(0)) == 1
    assert ctx.match(Plan.preset(24)) == 0


@pytest.mark.parametrize("q", [0, 24, 25, 1, 2])
def test_device_work_model_matches_oracle(g2, orc, ctx, q):
    from g2aimd.context import Plan
    g = g2.Graph.rmat(11, 16, seed=4).degeneracy_recoded()
    plan = Plan.preset(q)
    ctx.load(g)
    w = np.zeros(1, np.uint64)
    c = ctx.match(plan, work_bytes=w)
    want = orc.match(g, plan, threads=8)
    assert c == want["count"]
    assert int(w[0]) == want["work"]
    if plan.k > 2:
        w2 = np.zeros(1, np.uint64)
        assert ctx.match(plan, intersect_mode=1, work_bytes=w2) == want["count"]
        assert int(w2[0]) == want["work"]


@pytest.mark.parametrize("q,scale,ef", [(1, 12, 16), (2, 12, 16), (3, 10, 8), (9, 10, 8), (17, 9, 8)])
def test_plan_walk_handoff_keeps_counts(g2, orc, ctx, q, scale, ef):
    """Plan walks hand pending work (window halves, candidate batches, last-level
    scan halves) to idle warps; with hand-offs forced early (every 1000 SM
    cycles) and switched off, per-root counts and the work model stay the
    oracle's."""
    from g2aimd.context import Plan
    plan = Plan.preset(q)
    g = g2.Graph.rmat(scale, ef, seed=6).degeneracy_recoded()  # oracle sized to seconds
    ctx.load(g)
    want = orc.match(g, plan, threads=8, per_root=True)
    for kw in ({"spill_kcycles": 1}, {"spill_kcycles": 1, "schedule": "heuristic"}, {"flags": 16}):
        rc = np.zeros(g.n, np.uint64)
        assert ctx.match(plan, root_counts=rc, intersect_mode=1, **kw) == want["count"], (q, kw)
        assert np.array_equal(rc, want["root_counts"]), (q, kw)
        records, _ = ctx.spill_stats()
        assert (records == 0) == (kw.get("flags") == 16), (q, kw, records)
        w = np.zeros(1, np.uint64)
        ctx.match(plan, work_bytes=w, intersect_mode=1, **kw)
        assert int(w[0]) == want["work"], (q, kw)


def test_l2_persistence_window_keeps_counts(g2, orc, ctx):
    """The L2 persistence window (device-stream runs) changes nothing but cache policy."""
    import torch
    from g2aimd.context import Plan
    g = g2.Graph.rmat(12, 16, seed=3).degeneracy_recoded()
    ctx.load(g)
    out = torch.zeros(1, dtype=torch.int64, device="cuda:0")
    s = torch.cuda.Stream()  # the window is a stream attribute: not the legacy stream
    for q in (24, 1):
        plan = Plan.preset(q)
        ctx.set_plan(plan)
        ctx.match_device(out.data_ptr(), stream=s.cuda_stream, flags=32)
        s.synchronize()
        assert int(out[0].item()) == orc.match(g, plan, threads=8)["count"], q


@pytest.mark.parametrize("q", [2, 5, 7, 9, 11, 13])
def test_shared_last_position_small_slabs(g2, orc, q):
    """Plans whose last position has no back neighbour at the position before
    it (diamonds, presets 5, 7, 9-15) count it from one candidate set per
    prefix.  With 256 scratch words per warp (512 for k = 6) that set holds at
    most 64 entries (96 for k = 6): larger sets (the hubs' at k = 4, 5) take
    the per-candidate scan, the rest the shared set.  Per-root counts and the work
    model stay the oracle's, hand-off on and off."""
    from g2aimd.context import Context, Plan
    plan = Plan.preset(q)
    scale, ef, words = {4: (11, 16, 256), 5: (9, 16, 256), 6: (8, 8, 512)}[plan.k]
    g = g2.Graph.rmat(scale, ef, seed=8).degeneracy_recoded()
    want = orc.match(g, plan, threads=8, per_root=True)
    if q == 2:  # the heaviest edge's common neighbourhood exceeds the 64-entry set
        adj = [set(g.cols[g.row_ptrs[v]:g.row_ptrs[v + 1]].tolist()) for v in range(g.n)]
        top = np.argsort(-np.diff(g.row_ptrs.astype(np.int64)))[:2]
        assert len(adj[top[0]] & adj[top[1]]) > 64
    launch = dict(blocks=148, warps_per_block=8, intersect_mode=1)
    with Context(0, scratch_bytes=148 * 8 * words * 4) as c:
        c.load(g)
        for kw in ({}, {"spill_kcycles": 1}, {"flags": 16}):
            rc = np.zeros(g.n, np.uint64)
            assert c.match(plan, root_counts=rc, **launch, **kw) == want["count"], (q, kw)
            assert np.array_equal(rc, want["root_counts"]), (q, kw)
            w = np.zeros(1, np.uint64)
            c.match(plan, work_bytes=w, **launch, **kw)
            assert int(w[0]) == want["work"], (q, kw)


@pytest.mark.parametrize("k", [3, 4])
def test_shared_last_position_split_roots(g2, orc, ctx, k):
    """Wedges and 3-stars rooted at the centre (last position adjacent to the
    root only): with heavy roots split into parts, each part counts its own
    position-1 candidates against the shared set, so per-root sums stay the
    oracle's."""
    from g2aimd.context import Plan
    plan = Plan.from_edges(k, [(0, j) for j in range(1, k)])
    assert all(b == [0] for b in plan.to_dict()["bn"][1:])
    g = g2.Graph.rmat(11 if k == 3 else 9, 16, seed=9).degeneracy_recoded()
    want = orc.match(g, plan, threads=8, per_root=True)
    ctx.load(g)
    for kw in ({}, {"split": True, "schedule": "heuristic", "granularity": 64}, {"spill_kcycles": 1}):
        rc = np.zeros(g.n, np.uint64)
        assert ctx.match(plan, root_counts=rc, **kw) == want["count"], (k, kw)
        assert np.array_equal(rc, want["root_counts"]), (k, kw)


@pytest.mark.parametrize("words", [0, 256])
def test_cycle4_through_opposite_vertices(g2, orc, words):
    """4-cycles (preset 1): a root whose forward neighbours make the walk's
    per-pair intersections dearer than one count per id above the root
    (4 (ids spanned + the forward neighbours' degrees) <= (d - 1) x those
    degrees) counts every cycle through its vertex opposite the root.  Per-root counts equal the
    oracle's with the default slab and with 256-word slabs (up to six id ranges
    per root), in id and heuristic order, hand-off on and off."""
    from g2aimd.context import Context, Plan
    plan = Plan.preset(1)
    g = g2.Graph.rmat(12, 16, seed=11).degeneracy_recoded()
    rp = g.row_ptrs.astype(np.int64)
    deg = np.diff(rp)
    taken = 0  # roots that take the opposite-vertex count (the device's rule)
    for v in range(g.n):
        row = g.cols[rp[v]:rp[v + 1]]
        fw = row[row > v]
        nz = fw[deg[fw] > 0]
        if fw.size < 2 or nz.size == 0:
            continue
        xmax = int(max(g.cols[rp[y + 1] - 1] for y in nz))
        sdeg = int(deg[fw].sum())
        taken += xmax > v and 4 * ((xmax - v) + sdeg) <= (fw.size - 1) * sdeg
    assert 0 < taken < g.n
    want = orc.match(g, plan, threads=8, per_root=True)
    launch = dict(blocks=148, warps_per_block=8) if words else {}
    with Context(0, scratch_bytes=148 * 8 * words * 4) as c:
        c.load(g)
        for kw in ({}, {"schedule": "heuristic"}, {"flags": 16}):
            rc = np.zeros(g.n, np.uint64)
            assert c.match(plan, root_counts=rc, **launch, **kw) == want["count"], (words, kw)
            assert np.array_equal(rc, want["root_counts"]), (words, kw)
