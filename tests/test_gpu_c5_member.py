"""A scaled-down member of the C5 workload: the same device generator
(R-MAT a=.57 b=c=.19, edge factor 28) at scale 15, recoded on the device, with
the C5 jobs checked against the CPU oracle: every 4-clique, the 5-cliques of
the stride sample of roots the C5 leg uses (v % S == 0), and time-budgeted
maximal cliques over the roots that finished."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c5_small(g2):
    from g2aimd.context import Context, CostModel
    c = Context(0)
    m = c.gen_rmat(15, 28, seed=1)
    c.degeneracy_recode()
    c.set_model(CostModel.load(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                            "g2-aimd_b200", "models", "k4.npz")))
    g = c.copy_csr(m)
    yield c, g
    c.close()


def test_k4_all_roots(orc, c5_small):
    from g2aimd.context import Plan
    c, g = c5_small
    plan = Plan.preset(24)
    got = c.match(plan, schedule="heuristic", warps_per_block=4, chunk=1, ctas_per_sm=6)
    assert got == orc.match(g, plan, threads=os.cpu_count() or 1)["count"]
    assert c.match(plan, schedule="learned", flags=8, warps_per_block=4, chunk=1, ctas_per_sm=6) == got


def test_k5_stride_sample(orc, c5_small):
    from g2aimd.context import Plan
    c, g = c5_small
    plan = Plan.preset(25)
    roots = np.arange(0, g.n, 64, dtype=np.uint32)
    per = np.zeros(roots.size, np.uint64)
    got = c.match(plan, sources=roots, root_counts=per, schedule="heuristic")
    want = orc.match(g, plan, roots=roots, threads=os.cpu_count() or 1, per_root=True)
    assert got == want["count"]
    assert np.array_equal(per, want["root_counts"])


def test_budgeted_mce(orc, c5_small):
    c, g = c5_small
    count, hist, rn = c.mce(hist_len=512, root_nodes=True, deadline_ms=3)
    done = np.flatnonzero(rn > 0).astype(np.uint32)
    assert done.size > 0
    want = orc.mce(g, roots=done, hist_len=512, threads=os.cpu_count() or 1)
    assert count == want["count"] and np.array_equal(hist, want["hist"])
