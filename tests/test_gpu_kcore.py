"""Degeneracy order on the device equals the host order (core numbers and the
(core, degree, id) permutation), so either can prepare a graph for the kernels."""
import numpy as np
import pytest

from helpers import random_graph

pytestmark = pytest.mark.gpu


def test_device_order_equals_host_order(g2, ctx):
    graphs = [g2.Graph.from_edges(1, []), g2.Graph.from_edges(5, [(0, 1), (1, 2), (2, 0), (3, 4)]),
              random_graph(g2.Graph, 300, 0.05, 2, planted=[tuple(range(0, 60, 5))]),
              g2.Graph.rmat(14, 16, seed=3), g2.Graph.chung_lu(1 << 15, 2.2, 20.0, seed=9)]
    for g in graphs:
        perm_h, core_h = g.degeneracy_order()
        ctx.load(g)
        perm_d, core_d = ctx.degeneracy_order()
        assert np.array_equal(core_d, core_h), g.name
        assert np.array_equal(perm_d, perm_h), g.name


def recode_cases(g2):
    return [g2.Graph.from_edges(5, [(0, 1), (1, 2), (2, 0), (3, 4)]),
            random_graph(g2.Graph, 300, 0.05, 2, planted=[tuple(range(0, 60, 5))]),
            g2.Graph.rmat(13, 16, seed=3), g2.Graph.chung_lu(1 << 14, 2.2, 20.0, seed=9)]


def test_device_recode_equals_host_recode(g2, orc):
    """The recoded CSR, permutation and core numbers match the host's, and the
    context then enumerates the recoded graph (learned schedule included)."""
    from g2aimd.context import Context
    with Context(0) as c:
        for g in recode_cases(g2):
            want = g.degeneracy_recoded()
            perm_h, core_h = g.degeneracy_order()
            c.load(g)
            perm, core = c.degeneracy_recode()
            assert np.array_equal(perm, perm_h) and np.array_equal(core, core_h), g.name
            got = c.copy_csr(g.m)
            assert np.array_equal(got.row_ptrs, want.row_ptrs), g.name
            assert np.array_equal(got.cols, want.cols), g.name
            count, hist = c.mce(hist_len=64, schedule="heuristic")
            ref = orc.mce(want, hist_len=64)
            assert count == ref["count"] and np.array_equal(hist, ref["hist"]), g.name
            # core numbers are loaded under the new names: the learned features use them
            feats = c.root_features(np.arange(min(64, g.n), dtype=np.uint32))
            c.load(want)
            c.load_core(want.core)
            assert np.allclose(feats, c.root_features(np.arange(min(64, g.n), dtype=np.uint32))), g.name


def test_device_recode_in_chunks(g2, monkeypatch):
    """Rows sorted in several segmented-sort calls give the same CSR; a row longer
    than a call may hold is refused, not cut."""
    from g2aimd.context import Context
    g = g2.Graph.rmat(12, 8, seed=5)
    want = g.degeneracy_recoded()
    longest = int(np.diff(g.row_ptrs).max())
    with Context(0) as c:
        monkeypatch.setenv("G2_RECODE_CHUNK", str(longest + 7))
        c.load(g)
        c.degeneracy_recode()
        got = c.copy_csr(g.m)
        assert np.array_equal(got.row_ptrs, want.row_ptrs) and np.array_equal(got.cols, want.cols)
        monkeypatch.setenv("G2_RECODE_CHUNK", str(longest - 1))
        c.load(g)
        with pytest.raises(Exception, match="unsupported"):
            c.degeneracy_recode()
