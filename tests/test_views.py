"""Views for the out-of-core path, on the host (no GPU): the ball, the id
renumbering and the row rule of g2_view_materialize against a direct Python
construction; the radii a plan needs; and the property the pipeline rests on,
checked with the oracle: summing the searches rooted at each bin's sources over
its view gives the whole graph's answer (maximal cliques with their size
histogram, plan-driven matches of several queries)."""
import numpy as np
import pytest

from helpers import random_graph, small_graphs


def py_view(g, sources, radius, row_radius, min_deg, upper=False, forward=False, ego=False):
    """Direct construction: per kept source, BFS depths (through vertices above
    the source when upper); a vertex's depth is its smallest; ascending ids;
    rows of vertices within row_radius restricted to the ball (and to entries
    above the row's vertex when forward)."""
    rp, ci = g.row_ptrs, g.cols
    deg = np.diff(rp)
    kept = [int(s) for s in sources if deg[s] >= min_deg]
    depth = {}
    for s in set(kept):
        seen = {s: 0}
        frontier = [s]
        for d in range(radius):
            nxt = []
            for x in frontier:
                for u in ci[rp[x]:rp[x + 1]].tolist():
                    if u not in seen and (not upper or u > s):
                        seen[u] = d + 1
                        nxt.append(u)
            frontier = nxt
        for x, d in seen.items():
            depth[x] = min(depth.get(x, d), d)
    ids = sorted(depth)
    local = {g_: i for i, g_ in enumerate(ids)}
    # ego: the sources' closed neighbourhoods as seen in the (forward) rows
    hoods = []
    if ego:
        for s in set(kept):
            hoods.append({s} | {u for u in ci[rp[s]:rp[s + 1]].tolist() if u in local and (not forward or u > s)})
    rows = []
    for g_ in ids:
        if depth[g_] <= row_radius:
            row = [u for u in ci[rp[g_]:rp[g_ + 1]].tolist() if u in local and (not forward or u > g_)]
            if ego:
                row = [u for u in row if any(g_ in h and u in h for h in hoods)]
            rows.append([local[u] for u in row])
        else:
            rows.append([])
    return ids, rows, [local[s] for s in kept]


def check_view(g, sources, radius, row_radius, min_deg=0, upper=False, forward=False, ego=False):
    v, lsrc, ids = g.view(sources, radius=radius, row_radius=row_radius, min_root_degree=min_deg, upper=upper,
                          forward=forward, ego=ego)
    want_ids, want_rows, want_src = py_view(g, sources, radius, row_radius, min_deg, upper, forward, ego)
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
                for upper, forward in ((False, False), (True, False), (True, True), (False, True)):
                    check_view(g, src, radius, row_radius, min_deg=int(trial == 2) * 2, upper=upper,
                               forward=forward)


def test_view_structure_rmat(g2):
    g = g2.Graph.rmat(10, 8, seed=5)
    rng = np.random.default_rng(11)
    for radius, row_radius in ((1, 1), (2, 1), (2, 2)):
        for upper, forward in ((False, False), (True, False), (True, True)):
            src = rng.choice(g.n, size=40, replace=False)  # unsorted: upper walks sort them
            check_view(g, src, radius, row_radius, upper=upper, forward=forward)


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
    assert lib.g2_view_materialize(rp, ci, g.n, src.ctypes.data_as(C.c_void_p), 1, 1, 1, 0, 0, C.byref(v)) == -1
    src = np.array([0], np.uint32)
    sp = src.ctypes.data_as(C.c_void_p)
    assert lib.g2_view_materialize(rp, ci, g.n, sp, 1, 1, 2, 0, 0, C.byref(v)) == -1  # row radius > radius
    assert lib.g2_view_materialize(rp, ci, g.n, sp, 1, 1, 1, 0, 16, C.byref(v)) == -1  # unknown flag
    assert lib.g2_view_materialize(rp, ci, g.n, sp, 1, 1, 1, 0, 1, C.byref(v)) == 0
    lib.g2_view_free(C.byref(v))


def plan_shape_py(plan):
    """Distances from position 0 in the query graph of the plan's back
    neighbours; upper = every position provably above position 0."""
    r = plan.raw
    k = r.k
    adj = [set() for _ in range(k)]
    is_bn = [False] * k
    gt = set()  # (a, b): M(a) > M(b), positions
    for i in range(k):
        for j in range(r.bn_count[i]):
            p = r.id2order[r.bn[i][j]]
            adj[i].add(p)
            adj[p].add(i)
            is_bn[p] = True
        u = r.order[i]
        for j in range(r.cond_count[u]):
            op, w = r.cond[u][j][0], r.id2order[r.cond[u][j][1]]
            if op == 1:
                gt.add((i, w))
            elif op == 0:
                gt.add((w, i))
    changed = True
    while changed:
        extra = {(a, c) for (a, b) in gt for (b2, c) in gt if b == b2} - gt
        changed = bool(extra)
        gt |= extra
    upper = all((i, 0) in gt for i in range(1, k))
    forward = all((i, j) in gt for i in range(1, k) for j in range(i))
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
    return {"radius": max(dist.values()), "row_radius": max(dist[i] for i in range(k) if is_bn[i]),
            "min_root_degree": len(adj[0]), "upper": upper, "forward": forward}


@pytest.mark.parametrize("q", [0, 1, 2, 3, 4, 5, 6, 23, 24, 25])
def test_plan_view_shape(q):
    from g2aimd.context import Plan
    p = Plan.preset(q)
    sh = p.view_shape()
    assert sh == plan_shape_py(p)
    # the reference's single hop count covers the view's rows
    assert sh["row_radius"] <= p.raw.hop - 1 <= sh["radius"]
    assert sh["min_root_degree"] == p.raw.root_degree


def test_known_shapes():
    from g2aimd.context import Plan
    tri, c4, diamond, k4 = (Plan.preset(q).view_shape() for q in (0, 1, 2, 24))
    assert (tri["radius"], tri["row_radius"], tri["upper"]) == (1, 1, True)
    assert (c4["radius"], c4["row_radius"], c4["upper"]) == (2, 1, True)  # opposite corner at distance 2
    assert (diamond["radius"], diamond["upper"]) == (1, False)  # conditions only "!=" against the root
    assert (k4["radius"], k4["min_root_degree"], k4["upper"]) == (1, 3, True)
    assert tri["forward"] and k4["forward"] and not c4["forward"] and not diamond["forward"]


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
    sh = plan.view_shape()
    for nbins in (1, 5, 40):
        bin_of = np.random.default_rng(q * 100 + nbins).integers(0, nbins, g.n).astype(np.uint32)
        for upper, forward in sorted({(False, False), (sh["upper"], False), (sh["upper"], sh["forward"])}):
            total = 0
            for src in by_bin(bin_of, nbins):
                v, lsrc, _ = g.view(src, **dict(sh, upper=upper, forward=forward))
                if lsrc.size:
                    total += orc.match(v, plan, roots=lsrc)["count"]
            assert total == want, (q, nbins, upper, forward, total, want)


def test_upper_views_are_smaller(g2):
    """Where the query allows it, upper views skip everything below each source."""
    from g2aimd.context import Plan
    g = g2.Graph.rmat(11, 8, seed=3).degeneracy_recoded()
    sh = Plan.preset(24).view_shape()
    src = np.arange(0, g.n, 7, dtype=np.uint32)
    full, _, _ = g.view(src, **dict(sh, upper=False, forward=False))
    up, _, _ = g.view(src, **dict(sh, forward=False))
    fwd, _, _ = g.view(src, **sh)
    assert up.m < full.m and up.n < full.n
    assert fwd.n == up.n and 2 * fwd.m <= up.m  # each kept edge at most once


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


@pytest.mark.parametrize("radius,row_radius,upper,forward", [(1, 1, False, False), (2, 1, False, False),
                                                            (1, 1, True, False), (2, 1, True, False),
                                                            (2, 2, True, False), (1, 1, True, True),
                                                            (2, 2, False, True)])
def test_view_bins_respect_budget(g2, radius, row_radius, upper, forward):
    g = g2.Graph.rmat(10, 8, seed=9)
    budget = 48 << 10 if not forward else 24 << 10
    kw = dict(radius=radius, row_radius=row_radius, upper=upper, forward=forward)
    nb, bin_of = g.view_bins(max_bytes=budget, **kw)
    assert nb >= 2
    assert bin_of.max() == nb - 1
    assert np.all(np.diff(bin_of.astype(np.int64)) >= 0)  # ranges of ids, in order
    bins = by_bin(bin_of, nb)
    for b, src in enumerate(bins):
        assert src.size > 0
        v, lsrc, _ = g.view(src, **kw)
        size = view_bytes(v, lsrc.size)
        # the bin's view is counted exactly (up to the layout's alignment padding) ...
        assert src.size == 1 or size <= budget + 48
        # ... so the bin was closed because the next root did not fit
        if b + 1 < nb:
            v2, l2, _ = g.view(np.append(src, bins[b + 1][0]), **kw)
            assert view_bytes(v2, l2.size) > budget - 48
    nb_big, _ = g.view_bins(max_bytes=1 << 40, **kw)
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


@pytest.mark.parametrize("upper,forward", [(False, False), (True, False), (True, True)])
@pytest.mark.parametrize("step", [1, 2])
def test_large_views_built_by_threads_equal_one_thread(g2, monkeypatch, upper, forward, step):
    """Views of at least 2^14 vertices have their rows counted and written by
    several threads, and radius-1 balls of at least 2^14 roots are walked by
    them; the result is the one-thread view."""
    g = g2.Graph.rmat(15, 8, seed=12).degeneracy_recoded()
    src = np.arange(0, g.n, step, dtype=np.uint32)
    kw = dict(radius=1, row_radius=1, upper=upper, forward=forward)
    monkeypatch.setenv("G2_HOST_THREADS", "1")
    one, s1, i1 = g.view(src, **kw)
    monkeypatch.setenv("G2_HOST_THREADS", "6")
    many, s6, i6 = g.view(src, **kw)
    assert one.n >= 1 << 14
    assert np.array_equal(one.row_ptrs, many.row_ptrs) and np.array_equal(one.cols, many.cols)
    assert np.array_equal(one.fwd_offsets, many.fwd_offsets) and one.max_fwd == many.max_fwd
    assert np.array_equal(s1, s6) and np.array_equal(i1, i6)


def test_ego_view_structure(g2):
    """Ego rows: an entry (u, y) stays when some kept source s has u and y in N[s]
    (within the rows the other flags keep)."""
    rng = np.random.default_rng(8)
    graphs = small_graphs(g2.Graph) + [g2.Graph.rmat(9, 8, seed=2)]
    for g in graphs:
        for trial in range(3):
            k = int(rng.integers(0, max(1, g.n) + 1))
            src = rng.choice(g.n, size=min(k, g.n), replace=False) if g.n else np.zeros(0, np.uint32)
            for upper, forward in ((False, False), (True, False), (True, True)):
                check_view(g, src, 1, 1, min_deg=int(trial == 2), upper=upper, forward=forward, ego=True)


def test_ego_needs_radius_one(g2):
    g = g2.Graph.from_edges(3, [(0, 1), (1, 2)])
    with pytest.raises(Exception):
        g.view([0], radius=2, row_radius=1, ego=True)


@pytest.mark.parametrize("nbins", [1, 5, 23])
def test_ego_views_sum_to_whole_graph_mce(g2, orc, nbins):
    g = random_graph(g2.Graph, 400, 0.04, 31, planted=[tuple(range(0, 30, 3))]).degeneracy_recoded()
    want = orc.mce(g, hist_len=64)
    bin_of = np.random.default_rng(nbins).integers(0, nbins, g.n).astype(np.uint32)
    count, hist, induced, ego = 0, np.zeros(64, np.uint64), 0, 0
    for src in by_bin(bin_of, nbins):
        full, _, _ = g.view(src, radius=1, row_radius=1, min_root_degree=1)
        v, lsrc, _ = g.view(src, radius=1, row_radius=1, min_root_degree=1, ego=True)
        induced += full.m
        ego += v.m
        if lsrc.size:
            got = orc.mce(v, roots=lsrc, hist_len=64)
            count += got["count"]
            hist += got["hist"]
    assert count == want["count"] and np.array_equal(hist, want["hist"])
    if nbins > 1:
        assert ego < induced


@pytest.mark.parametrize("q", [0, 2, 24, 25])
def test_ego_views_sum_to_whole_graph_match(g2, orc, q):
    from g2aimd.context import Plan
    g = random_graph(g2.Graph, 300, 0.05, 21, planted=[tuple(range(0, 24, 2))]).degeneracy_recoded()
    plan = Plan.preset(q)
    sh = plan.view_shape()
    assert sh["radius"] == 1
    want = orc.match(g, plan)["count"]
    for nbins in (1, 7):
        bin_of = np.random.default_rng(nbins).integers(0, nbins, g.n).astype(np.uint32)
        total = 0
        for src in by_bin(bin_of, nbins):
            v, lsrc, _ = g.view(src, ego=True, **sh)
            if lsrc.size:
                total += orc.match(v, plan, roots=lsrc)["count"]
        assert total == want, (q, nbins)


def test_large_ego_views_threads_equal_one_thread(g2, monkeypatch):
    g = g2.Graph.chung_lu(1 << 15, 2.3, 12.0, seed=4).degeneracy_recoded()
    src = np.arange(0, g.n, 3, dtype=np.uint32)
    monkeypatch.setenv("G2_HOST_THREADS", "1")
    one, _, _ = g.view(src, radius=1, row_radius=1, min_root_degree=1, ego=True)
    monkeypatch.setenv("G2_HOST_THREADS", "6")
    many, _, _ = g.view(src, radius=1, row_radius=1, min_root_degree=1, ego=True)
    assert np.array_equal(one.row_ptrs, many.row_ptrs) and np.array_equal(one.cols, many.cols)
    assert np.array_equal(one.fwd_offsets, many.fwd_offsets) and one.max_fwd == many.max_fwd


@pytest.mark.parametrize("upper,forward", [(False, False), (True, True)])
def test_parallel_bin_plan(g2, monkeypatch, upper, forward):
    """Graphs of >= 2^16 vertices are planned in contiguous root ranges on
    several threads: bins stay contiguous and within budget, and each range
    boundary costs at most one bin."""
    g = g2.Graph.chung_lu(1 << 17, 2.3, 10.0, seed=6).degeneracy_recoded()
    kw = dict(radius=1, row_radius=1, min_root_degree=1, upper=upper, forward=forward)
    budget = (g.row_ptrs.nbytes + g.cols.nbytes) // 40
    monkeypatch.setenv("G2_HOST_THREADS", "1")
    n1, b1 = g.view_bins(budget, **kw)
    monkeypatch.setenv("G2_HOST_THREADS", "6")
    n6, b6 = g.view_bins(budget, **kw)
    assert n1 <= n6 <= n1 + 5
    for bins, nb in ((b1, n1), (b6, n6)):
        assert bins.max() == nb - 1 and np.all(np.diff(bins.astype(np.int64)) >= 0)
        for b in sorted(set(np.linspace(0, nb - 1, 12).astype(int).tolist())):
            src = np.flatnonzero(bins == b).astype(np.uint32)
            v, lsrc, _ = g.view(src, **kw)
            assert lsrc.size <= 1 or view_bytes(v, lsrc.size) <= budget + 48


def py_rebalance(g, bin_of, nbins, devices, times, reorder):
    """view/view_bin_manager.h:95-184 restated: Split (cut the bin furthest above
    the mean factor, roots alternately by descending degree, halves appended)
    then, as after Split or with Reorder, bins by descending factor."""
    deg = np.diff(g.row_ptrs).astype(np.int64)
    bins = [[v for v in range(g.n) if bin_of[v] == b] for b in range(nbins)]
    fac = lambda b: int(sum(deg[v] for v in b))  # noqa: E731
    if times:
        target = (nbins // devices + times) * devices
        while len(bins) < target:
            avg = sum(fac(b) for b in bins) // len(bins)
            pick, best = 0, 0
            for i, b in enumerate(bins):
                if fac(b) >= avg and fac(b) - avg > best:
                    pick, best = i, fac(b) - avg
            src = sorted(bins.pop(pick), key=lambda v: -deg[v])  # stable: ties by id
            bins += [src[1::2], src[0::2]]
    if times or reorder:
        bins = sorted(bins, key=lambda b: -fac(b))  # stable
    out = np.full(g.n, 0xFFFFFFFF, np.uint32)
    for k, b in enumerate(bins):
        out[b] = k
    return len(bins), out


@pytest.mark.parametrize("devices,times,reorder", [(1, 0, True), (4, 1, False), (3, 2, True), (8, 1, False)])
def test_rebalance_bins_follows_the_reference(g2, devices, times, reorder):
    g = g2.Graph.chung_lu(3000, 2.2, 10.0, seed=3).degeneracy_recoded()
    nb, bins = g.view_bins(40 << 10, radius=1, row_radius=1, min_root_degree=1)
    bins[::13] = 0xFFFFFFFF  # some vertices are no roots
    got = g.rebalance_bins(bins, nb, devices, times, reorder)
    want = py_rebalance(g, bins, nb, devices, times, reorder)
    assert got[0] == want[0] and np.array_equal(got[1], want[1])
    if times:
        assert got[0] == (nb // devices + times) * devices
    # the roots and their partition into bins are kept, only relabelled or cut
    assert np.array_equal(got[1] == 0xFFFFFFFF, bins == 0xFFFFFFFF)
