"""Hang guard of the hand-off record queue: every wait of a warp for a record
is bounded (g2_opts.wait_cycles, default 2^37 SM cycles).  With the bound cut
to one cycle the warps that wait give up, the run reports G2_ERR_TIMEOUT (a
status word the host reads, no device fault), and the same context then runs
normally."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G2_ERR_TIMEOUT = -4


def test_mce_wait_limit_reports_timeout_then_context_recovers(orc, c1_graph):
    from g2aimd._lib import G2Error
    from g2aimd.context import Context
    g = c1_graph
    want = orc.mce(g, hist_len=64)
    with Context(0) as c:
        c.load(g)
        with pytest.raises(G2Error) as err:
            c.mce(hist_len=64, wait_cycles=1, spill_kcycles=1)
        assert err.value.code == G2_ERR_TIMEOUT
        count, hist = c.mce(hist_len=64)
        assert count == want["count"] and np.array_equal(hist, want["hist"])


def test_plan_walk_wait_limit_reports_timeout_then_context_recovers(orc, g2):
    from g2aimd._lib import G2Error
    from g2aimd.context import Context, Plan
    g = g2.Graph.rmat(10, 12, seed=6).degeneracy_recoded()
    plan = Plan.preset(1)  # 4-cycles: the generic plan walk, which hands work off
    want = orc.match(g, plan, threads=4)["count"]
    with Context(0) as c:
        c.load(g)
        with pytest.raises(G2Error) as err:
            c.match(plan, wait_cycles=1, spill_kcycles=1)
        assert err.value.code == G2_ERR_TIMEOUT
        assert c.match(plan) == want
