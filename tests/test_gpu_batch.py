"""Batches of graphs in one launch per job (g2_batch_load / g2_batch_mce /
g2_batch_match): per-graph counts equal the oracle's on each graph alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(g2):
    from g2aimd.graph import chung_lu_batch
    gs = chung_lu_batch(count=9, seed=5, n_range=(300, 3000), degree_range=(4.0, 16.0))
    gs.append(g2.Graph.er(400, 0.05, planted=2, planted_size=9, seed=3).degeneracy_recoded())
    gs.append(g2.Graph.from_edges(4, []))  # an edgeless member
    return gs


def test_batch_mce_per_graph(g2, orc, ctx):
    gs = _batch(g2)
    ctx.batch_load(gs)
    want = [orc.mce(g, threads=4, hist_len=64) for g in gs]
    for kw in ({}, {"schedule": "heuristic"}, {"flags": 16}, {"spill_kcycles": 1}):
        counts, hist = ctx.batch_mce(hist_len=64, **kw)
        assert [int(c) for c in counts] == [w["count"] for w in want], kw
        assert np.array_equal(hist, np.sum([w["hist"] for w in want], axis=0)), kw


@pytest.mark.parametrize("q", [0, 1, 2, 24])
def test_batch_match_per_graph(g2, orc, ctx, q):
    from g2aimd.context import Plan
    gs = _batch(g2)
    ctx.batch_load(gs)
    plan = Plan.preset(q)
    want = [orc.match(g, plan, threads=4)["count"] for g in gs]
    for kw in ({}, {"schedule": "heuristic", "split": True, "granularity": 64}):
        assert [int(c) for c in ctx.batch_match(plan, **kw)] == want, (q, kw)


def test_single_graph_load_clears_batch(g2, ctx):
    gs = _batch(g2)
    ctx.batch_load(gs)
    ctx.load(gs[0])
    with pytest.raises(g2.G2Error):
        ctx.batch_mce()
