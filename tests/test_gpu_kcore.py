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
