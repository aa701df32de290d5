"""Runs captured in a CUDA graph and replayed: the device-stream entry points
enqueue only stream work once their buffers exist, and every run (replay
included) bumps the hand-off epoch on the device, so records of an earlier
replay never look published.  Counts stay the oracle's on every replay."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_cuda_graph_replays_mce_and_plan_walk(g2, orc):
    import torch
    from g2aimd.context import Context, Plan
    g = g2.Graph.rmat(11, 16, seed=2).degeneracy_recoded()
    want_mce = orc.mce(g, threads=8, hist_len=64)
    plan = Plan.preset(1)  # 4-cycles: the plan walk with hand-off
    want_c4 = orc.match(g, plan, threads=8)["count"]
    with Context(0) as ctx:
        ctx.load(g)
        ctx.set_plan(plan)
        s = torch.cuda.Stream()
        out_m = torch.zeros(1 + 64, dtype=torch.int64, device="cuda:0")
        out_p = torch.zeros(1, dtype=torch.int64, device="cuda:0")

        def step():  # hand-offs forced early so that records are written on every replay
            ctx.mce_device(out_m.data_ptr(), 64, stream=s.cuda_stream, spill_kcycles=1)
            ctx.match_device(out_p.data_ptr(), stream=s.cuda_stream, spill_kcycles=1)

        with torch.cuda.stream(s):
            step()  # allocates every buffer the runs need
        s.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s, capture_error_mode="relaxed"):
            step()
        for _ in range(3):
            out_m.fill_(-1)
            out_p.fill_(-1)
            graph.replay()
            torch.cuda.synchronize()
            assert int(out_m[0]) == want_mce["count"]
            assert np.array_equal(out_m[1:].cpu().numpy().astype(np.uint64), want_mce["hist"])
            assert int(out_p[0]) == want_c4
        del graph
