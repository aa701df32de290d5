"""MCE with a time budget (g2_opts.deadline_ms): past the budget warps start no
new root and drop the root they walk, so the run ends soon after and returns
G2_ERR_DEADLINE with the results of the roots that finished.  Those results are
exact: the count and histogram equal the oracle's over exactly the roots whose
search-tree node count is non-zero.  The limit is a device clock read, not a
fault: the context stays usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_generous_budget_changes_nothing(orc, c1_graph):
    from g2aimd.context import Context
    g = c1_graph
    want = orc.mce(g, hist_len=64)
    with Context(0) as c:
        c.load(g)
        count, hist, _rn = c.mce(hist_len=64, root_nodes=True, deadline_ms=60000)
        assert not c.expired
        assert count == want["count"] and np.array_equal(hist, want["hist"])


def test_budget_run_out_keeps_finished_roots_exact(g2, orc):
    from g2aimd.context import Context
    g = g2.Graph.rmat(14, 16, seed=1).degeneracy_recoded()
    with Context(0) as c:
        c.load(g)
        count, hist, rn = c.mce(hist_len=128, root_nodes=True, deadline_ms=5)
        assert c.expired
        done = np.flatnonzero(rn > 0).astype(np.uint32)
        assert 0 < done.size < g.n
        want = orc.mce(g, roots=done, hist_len=128, threads=8)
        assert count == want["count"] and np.array_equal(hist, want["hist"])
        # the context runs normally afterwards
        c2, _h2 = c.mce(sources=done[:256], hist_len=128)
        assert c2 == orc.mce(g, roots=done[:256], hist_len=128)["count"] and not c.expired


@pytest.mark.parametrize("q,budget", [(24, 1), (25, 2), (1, 5), (2, 5)])
def test_match_budget_keeps_finished_roots_exact(g2, orc, q, budget):
    """Plan-driven counts with a time budget: clique plans (bitmap path) and
    plan walks (4-cycles, diamonds).  Finished roots are the ones with a
    recorded cost; the count equals the oracle's over exactly those roots."""
    from g2aimd.context import Context, Plan
    g = g2.Graph.rmat(16, 16, seed=3).degeneracy_recoded()
    plan = Plan.preset(q)
    with Context(0) as c:
        c.load(g)
        c.load_core(g.core)
        full = c.match(plan, schedule="heuristic", flags=1)
        cost = np.zeros(g.n, np.uint64)
        got = c.match(plan, root_cost=cost, schedule="heuristic", flags=1, deadline_ms=budget)
        done = np.flatnonzero(cost > 0).astype(np.uint32)
        if c.expired:
            assert done.size < g.n and got <= full
        else:
            assert got == full
        want = orc.match(g, plan, roots=done, threads=8)["count"]
        assert got == want
        # generous budget: everything finishes
        assert c.match(plan, schedule="heuristic", flags=1, deadline_ms=600000) == full and not c.expired


def test_device_stream_status_reports_the_budget(g2):
    """g2_run_status gives a device-stream run's outcome: G2_ERR_DEADLINE when
    its budget ran out before every root finished (a run that takes more than
    ten times the budget), 0 for a run without one."""
    import torch
    from g2aimd.context import Context, Plan
    g = g2.Graph.rmat(16, 16, seed=3).degeneracy_recoded()
    dev = torch.device("cuda", 0)
    st = torch.cuda.Stream(dev)
    out = torch.zeros(1, dtype=torch.int64, device=dev)
    with Context(0) as c:
        c.load(g)
        c.load_core(g.core)
        c.set_plan(Plan.preset(1))  # 4-cycles: the plan walk
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        c.match_device(out.data_ptr(), stream=st.cuda_stream, schedule="heuristic", flags=1)
        e1.record(st)
        assert c.run_status(st.cuda_stream) == 0
        full, full_ms = int(out[0].item()), e0.elapsed_time(e1)
        c.match_device(out.data_ptr(), stream=st.cuda_stream, schedule="heuristic", flags=1, deadline_ms=1)
        code = c.run_status(st.cuda_stream)
        if full_ms > 10.0:
            assert code == -11 and int(out[0].item()) < full  # G2_ERR_DEADLINE
        else:
            assert code in (0, -11)
