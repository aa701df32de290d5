"""The CPU oracle against independent brute force and the reference planner's
own output (no GPU)."""
import json
import os

import numpy as np
import pytest

from helpers import random_graph, small_graphs

HERE = os.path.dirname(os.path.abspath(__file__))


def golden_plans():
    with open(os.path.join(HERE, "golden", "plans.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("ref", golden_plans(), ids=lambda r: f"q{r['query']}")
def test_plan_oracle_matches_reference_planner(ref):
    import plan_oracle
    mine = plan_oracle.preset_plan(ref["query"])
    for key, val in ref.items():
        assert mine[key] == val, (ref["query"], key)


def test_mce_oracle_vs_bruteforce(g2, orc):
    for g in small_graphs(g2.Graph):
        want_c, want_h = orc.mce_bruteforce(g, 64)
        got = orc.mce(g, hist_len=64)
        assert got["count"] == want_c, g.name
        assert np.array_equal(got["hist"], want_h), g.name


def test_mce_oracle_hand_counts(g2, orc):
    G = g2.Graph
    assert orc.mce(G.from_edges(5, []))["count"] == 0          # isolated vertices are skipped
    assert orc.mce(G.from_edges(2, [(0, 1)]))["count"] == 1
    assert orc.mce(G.from_edges(4, [(0, 1), (1, 2), (2, 3)]))["count"] == 3
    r = orc.mce(G.from_edges(5, [(a, b) for a in range(5) for b in range(a + 1, 5)]))
    assert r["count"] == 1 and r["hist"][5] == 1
    # C4: four maximal edges
    assert orc.mce(G.from_edges(4, [(0, 1), (1, 2), (2, 3), (3, 0)]))["count"] == 4


def test_mce_oracle_thread_invariance(g2, orc):
    g = random_graph(g2.Graph, 300, 0.08, 5, planted=[tuple(range(0, 120, 10))]).degeneracy_recoded()
    a = orc.mce(g, threads=1, per_root=True)
    b = orc.mce(g, threads=4, per_root=True)
    assert a["count"] == b["count"] and np.array_equal(a["hist"], b["hist"])
    assert np.array_equal(a["root_nodes"], b["root_nodes"]) and a["work"] == b["work"]


@pytest.mark.parametrize("q", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 16, 23, 24, 25])
def test_match_oracle_vs_embeddings(g2, orc, q):
    import plan_oracle
    from g2aimd.context import Plan
    k, edges = plan_oracle.PRESETS[q]
    aut = plan_oracle.aut_size(k, edges)
    plan = Plan.preset(q)
    for s, g in enumerate([random_graph(g2.Graph, 14, 0.45, 7 + q), random_graph(g2.Graph, 18, 0.3, 70 + q,
                                                                                  planted=[(0, 1, 2, 3, 4, 5)])]):
        emb = orc.embeddings(g, k, edges)
        assert emb % aut == 0
        assert orc.match(g, plan)["count"] == emb // aut, (q, s)


def test_kcore_oracle_vs_library_order(g2, orc):
    g = g2.Graph.rmat(12, 8, seed=3)
    order, core, kmax = orc.kcore(g)
    perm, core2 = g.degeneracy_order()
    assert np.array_equal(core, core2)
    # new ids are sorted by (core, degree): check monotone along the new order
    inv = np.argsort(perm)
    c = core2[inv].astype(np.int64)
    d = g.degrees()[inv]
    assert np.all(np.diff(c) >= 0)
    same = np.diff(c) == 0
    assert np.all(np.diff(d)[same] >= 0)
    assert kmax == int(core.max())


def test_oracle_builds_the_librarys_rmat_graphs(g2, orc):
    """The CPU measurement of the reference algorithm builds its input without
    the library: the oracle's generator and kcore-order recode give the same CSR
    (and core numbers) as g2_gen_rmat + the library's recode."""
    for scale, ef, seed in ((8, 8, 1), (12, 16, 3), (13, 28, 5)):
        o = orc.degeneracy_recoded(orc.gen_rmat(scale, ef, seed=seed))
        g = g2.Graph.rmat(scale, ef, seed=seed).degeneracy_recoded()
        assert np.array_equal(o.row_ptrs, g.row_ptrs)
        assert np.array_equal(o.cols, g.cols)
        assert np.array_equal(o.core, g.core)


def test_oracle_preset_plans_equal_the_librarys(g2, orc):
    from g2aimd.context import Plan
    for q in (0, 1, 2, 23, 24, 25):
        a, b = orc.PresetPlan(q), Plan.preset(q)
        assert a.k == b.k
        assert all(np.array_equal(x, y) for x, y in zip(a.flat(), b.flat()))


def _adjacency(g):
    rp = g.row_ptrs.astype(np.int64)
    return [g.cols[rp[v]:rp[v + 1]].astype(np.int64) for v in range(g.n)]


@pytest.mark.parametrize("seed", [11, 12])
def test_cycle4_count_through_opposite_vertices(g2, orc, seed):
    """The identity behind the GPU's opposite-vertex 4-cycle count: for the
    4-cycle plan, the oracle's count of root v equals the sum over x > v of
    C(c_x, 2), c_x = the neighbours y > v of v adjacent to x."""
    from g2aimd.context import Plan
    g = g2.Graph.rmat(10, 16, seed=seed).degeneracy_recoded()
    want = orc.match(g, Plan.preset(1), threads=4, per_root=True)["root_counts"]
    adj = _adjacency(g)
    got = np.zeros(g.n, np.uint64)
    for v in range(g.n):
        fw = adj[v][adj[v] > v]
        if fw.size < 2:
            continue
        xs = np.concatenate([adj[y][adj[y] > v] for y in fw])
        c = np.bincount(xs - v - 1) if xs.size else np.zeros(0, np.int64)
        got[v] = int((c * (c - 1) // 2).sum())
    assert np.array_equal(got, want)


@pytest.mark.parametrize("seed", [11, 12])
def test_diamond_count_from_one_shared_set(g2, orc, seed):
    """The identity behind the GPU's shared last-position set for diamonds
    (positions 2 and 3 share their candidates): the oracle's count of root v
    equals the sum over neighbours u > v of C(|N(v) & N(u)|, 2)."""
    from g2aimd.context import Plan
    g = g2.Graph.rmat(10, 16, seed=seed).degeneracy_recoded()
    want = orc.match(g, Plan.preset(2), threads=4, per_root=True)["root_counts"]
    adj = _adjacency(g)
    got = np.zeros(g.n, np.uint64)
    for v in range(g.n):
        for u in adj[v][adj[v] > v]:
            s = np.intersect1d(adj[v], adj[u], assume_unique=True).size
            got[v] += s * (s - 1) // 2
    assert np.array_equal(got, want)
