"""Views for the out-of-core path, on the host (no GPU): the ball, the id
renumbering and the row rule of g2_view_materialize against a direct Python
construction; the radii a plan needs; and the property the pipeline rests on,
checked with the oracle: summing the searches rooted at each bin's sources over
its view gives the whole graph's answer (maximal cliques with their size
histogram, plan-driven matches of several queries)."""
import numpy as np
import pytest

from helpers import random_graph, small_graphs


def py_view(g, sources, radius, row_radius, min_deg):
    """Direct construction: BFS depths from the kept sources, ascending ids,
    rows of vertices within row_radius restricted to the ball."""
    rp, ci = g.row_ptrs, g.cols
    deg = np.diff(rp)
    kept = [int(s) for s in sources if deg[s] >= min_deg]
    depth = {}
    frontier = []
    for s in kept:
        if s not in depth:
            depth[s] = 0
            frontier.append(s)
    for d in range(radius):
        nxt = []
        for x in frontier:
            for u in ci[rp[x]:rp[x + 1]].tolist():
                if u not in depth:
                    depth[u] = d + 1
                    nxt.append(u)
        frontier = nxt
    ids = sorted(depth)
    local = {g_: i for i, g_ in enumerate(ids)}
    rows = []
    for g_ in ids:
        if depth[g_] <= row_radius:
            rows.append([local[u] for u in ci[rp[g_]:rp[g_ + 1]].tolist() if u in local])
        else:
            rows.append([])
    return ids, rows, [local[s] for s in kept]


def check_view(g, sources, radius, row_radius, min_deg=0):
    v, lsrc, ids = g.view(sources, radius=radius, row_radius=row_radius, min_root_degree=min_deg)
    want_ids, want_rows, want_src = py_view(g, sources, radius, row_radius, min_deg)
    assert ids.tolist() == want_ids
    assert lsrc.tolist() == want_src
    assert v.n == len(want_ids) and v.row_ptrs[0] == 0
    max_fwd = 0
    for i, row in enumerate(want_rows):
        got = v.cols[v.row_ptrs[i]:v.row_ptrs[i + 1]].tolist()
        assert got == row, (i, got, row)
        assert v.fwd_offsets[i] == sum(1 for u in row if u <= i)
        max_fwd = max(max_fwd, len(row) - int(v.fwd_offsets[i]))
    assert v.max_fwd == max_fwd
    return v, lsrc


def test_view_structure_small_graphs(g2):
    rng = np.random.default_rng(3)
    for g in small_graphs(g2.Graph):
        for radius, row_radius in ((1, 1), (2, 1), (2, 2), (3, 1)):
            for trial in range(3):
                k = int(rng.integers(0, max(1, g.n) + 1))
                src = rng.choice(g.n, size=min(k, g.n), replace=False) if g.n else np.zeros(0, np.uint32)
                check_view(g, src, radius, row_radius, min_deg=int(trial == 2) * 2)


def test_view_structure_rmat(g2):
    g = g2.Graph.rmat(10, 8, seed=5)
    rng = np.random.default_rng(11)
    for radius, row_radius in ((1, 1), (2, 1), (2, 2)):
        src = np.sort(rng.choice(g.n, size=40, replace=False))
        check_view(g, src, radius, row_radius)


def test_view_duplicates_and_empty(g2):
    g = g2.Graph.from_edges(5, [(0, 1), (1, 2), (2, 0), (3, 4)])
    v, lsrc = check_view(g, [2, 2, 0], 1, 1)
    assert lsrc.tolist() == [2, 2, 0]
    v, lsrc = check_view(g, [], 1, 1)
    assert v.n == 0 and v.m == 0 and lsrc.size == 0
    v, lsrc = check_view(g, [3], 1, 1, min_deg=2)  # degree 1 < 2: dropped
    assert v.n == 0 and lsrc.size == 0


def test_view_rejects_bad_arguments(g2):
    import ctypes as C
    from g2aimd._lib import G2View
    g = g2.Graph.from_edges(3, [(0, 1), (1, 2)])
    src = np.array([5], np.uint32)  # out of range
    v = G2View()
    lib = g2.lib()
    rp, ci = g.row_ptrs.ctypes.data_as(C.c_void_p), g.cols.ctypes.data_as(C.c_void_p)
    assert lib.g2_view_materialize(rp, ci, g.n, src.ctypes.data_as(C.c_void_p), 1, 1, 1, 0, C.byref(v)) == -1
    src = np.array([0], np.uint32)
    assert lib.g2_view_materialize(rp, ci, g.n, src.ctypes.data_as(C.c_void_p), 1, 1, 2, 0, C.byref(v)) == -1


def plan_radii_py(plan):
    """Distances from position 0 in the query graph of the plan's back neighbours."""
    r = plan.raw
    k = r.k
    adj = [set() for _ in range(k)]
    is_bn = [False] * k
    for i in range(k):
        for j in range(r.bn_count[i]):
            p = r.id2order[r.bn[i][j]]
            adj[i].add(p)
            adj[p].add(i)
            is_bn[p] = True
    dist = {0: 0}
    fr = [0]
    while fr:
        nxt = []
        for x in fr:
            for y in adj[x]:
                if y not in dist:
                    dist[y] = dist[x] + 1
                    nxt.append(y)
        fr = nxt
    return max(dist.values()), max(dist[i] for i in range(k) if is_bn[i]), len(adj[0])


@pytest.mark.parametrize("q", [0, 1, 2, 3, 4, 5, 6, 23, 24, 25])
def test_plan_view_radius(q):
    from g2aimd.context import Plan
    p = Plan.preset(q)
    assert p.view_radius() == plan_radii_py(p)
    # the reference's single hop count covers the view's rows
    radius, row_radius, root_degree = p.view_radius()
    assert row_radius <= p.raw.hop - 1 <= radius
    assert root_degree == p.raw.root_degree


def test_known_radii():
    from g2aimd.context import Plan
    assert Plan.preset(0).view_radius() == (1, 1, 2)   # triangle
    assert Plan.preset(1).view_radius() == (2, 1, 2)   # 4-cycle: opposite corner at distance 2
    assert Plan.preset(24).view_radius() == (1, 1, 3)  # 4-clique


def bins_from_bounds(n, bounds):
    bin_of = np.zeros(n, np.uint32)
    for b, (lo, hi) in enumerate(zip(bounds[:-1], bounds[1:])):
        bin_of[lo:hi] = b
    return bin_of


def by_bin(bin_of, nbins):
    return [np.flatnonzero(bin_of == b).astype(np.uint32) for b in range(nbins)]


@pytest.mark.parametrize("nbins", [1, 3, 17])
def test_views_sum_to_whole_graph_mce(g2, orc, c1_graph, nbins):
    g = c1_graph
    want = orc.mce(g, hist_len=64)
    rng = np.random.default_rng(nbins)
    bin_of = rng.integers(0, nbins, g.n).astype(np.uint32)
    count, hist = 0, np.zeros(64, np.uint64)
    for src in by_bin(bin_of, nbins):
        v, lsrc, _ = g.view(src, radius=1, row_radius=1, min_root_degree=1)
        if lsrc.size == 0:
            continue
        got = orc.mce(v, roots=lsrc, hist_len=64)
        count += got["count"]
        hist += got["hist"]
    assert count == want["count"]
    assert np.array_equal(hist, want["hist"])


def test_views_sum_to_whole_graph_mce_rmat(g2, orc):
    g = g2.Graph.rmat(11, 8, seed=2).degeneracy_recoded()
    want = orc.mce(g, hist_len=64)
    nb, bin_of = g.view_bins(max_bytes=64 << 10, radius=1, row_radius=1, min_root_degree=1)
    assert nb > 4
    count, hist = 0, np.zeros(64, np.uint64)
    for src in by_bin(bin_of, nb):
        v, lsrc, _ = g.view(src, radius=1, row_radius=1, min_root_degree=1)
        if lsrc.size:
            got = orc.mce(v, roots=lsrc, hist_len=64)
            count += got["count"]
            hist += got["hist"]
    assert count == want["count"] and np.array_equal(hist, want["hist"])


@pytest.mark.parametrize("q", [0, 1, 2, 3, 24, 25])
def test_views_sum_to_whole_graph_match(g2, orc, q):
    from g2aimd.context import Plan
    g = random_graph(g2.Graph, 300, 0.05, 21, planted=[tuple(range(0, 24, 2))]).degeneracy_recoded()
    plan = Plan.preset(q)
    want = orc.match(g, plan)["count"]
    radius, row_radius, root_degree = plan.view_radius()
    for nbins in (1, 5, 40):
        bin_of = np.random.default_rng(q * 100 + nbins).integers(0, nbins, g.n).astype(np.uint32)
        total = 0
        for src in by_bin(bin_of, nbins):
            v, lsrc, _ = g.view(src, radius=radius, row_radius=row_radius, min_root_degree=root_degree)
            if lsrc.size:
                total += orc.match(v, plan, roots=lsrc)["count"]
        assert total == want, (q, nbins, total, want)


def test_view_too_small_radius_misses_matches(g2, orc):
    """The radii are needed: a 4-cycle's opposite corner lies at distance 2."""
    from g2aimd.context import Plan
    g = random_graph(g2.Graph, 200, 0.06, 5)
    plan = Plan.preset(1)
    want = orc.match(g, plan)["count"]
    assert want > 0
    src = np.arange(g.n, dtype=np.uint32)
    v, lsrc, _ = g.view(src[:50], radius=1, row_radius=1)
    short = orc.match(v, plan, roots=lsrc)["count"]
    v, lsrc, _ = g.view(src[:50], radius=2, row_radius=1)
    full = orc.match(v, plan, roots=lsrc)["count"]
    assert short < full == orc.match(g, plan, roots=src[:50])["count"]


def view_bytes(v, nsrc):
    a16 = lambda x: (x + 15) // 16 * 16  # noqa: E731
    fo = a16(8 * (v.n + 1))
    ci = a16(fo + 4 * v.n)
    src = a16(ci + 4 * v.m)
    return a16(src + 4 * nsrc)


@pytest.mark.parametrize("radius,row_radius", [(1, 1), (2, 1)])
def test_view_bins_respect_budget(g2, radius, row_radius):
    g = g2.Graph.rmat(10, 8, seed=9)
    budget = 48 << 10
    nb, bin_of = g.view_bins(max_bytes=budget, radius=radius, row_radius=row_radius)
    assert nb >= 2
    assert bin_of.max() == nb - 1
    assert np.all(np.diff(bin_of.astype(np.int64)) >= 0)  # ranges of ids, in order
    for src in by_bin(bin_of, nb):
        assert src.size > 0
        v, lsrc, _ = g.view(src, radius=radius, row_radius=row_radius)
        # the estimate bounds the view (up to the layout's alignment padding)
        assert src.size == 1 or view_bytes(v, lsrc.size) <= budget + 48
    nb_big, _ = g.view_bins(max_bytes=1 << 40, radius=radius, row_radius=row_radius)
    assert nb_big == 1


def test_view_bins_isolated_and_rejects(g2):
    g = g2.Graph.from_edges(4, [])
    nb, bins = g.view_bins(1 << 20, min_root_degree=1)  # no root has a neighbour
    assert nb == 1 and bins.tolist() == [0, 0, 0, 0]
    nb, bins = g.view_bins(1, min_root_degree=0)  # every root alone in its bin
    assert nb == 4 and bins.tolist() == [0, 1, 2, 3]
    g = g2.Graph.from_edges(3, [(0, 1)])
    with pytest.raises(Exception):
        g.view_bins(1 << 20, radius=1, row_radius=2)
