"""g2_match_count_noalloc: the count that allocates no device memory.

Callers that cannot let a library call cudaMalloc (their device memory belongs
to their own allocator or a fixed budget, or a cudaMalloc would synchronise a
latency-critical loop) use this entry point; it keeps its scratch in a static
device array.  Here it is called through the C ABI, twice in a row, and its
count is compared with the allocating entry point g2_match_run (integer
counts: exact equality).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib):
    f = lib.g2_match_count_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


@pytest.mark.parametrize("query", [24, 2])
def test_noalloc_matches_allocating_entry_point(g2, query):
    import torch

    from g2aimd.context import Context, Plan
    g = g2.Graph.rmat(12, 16, seed=17).degeneracy_recoded()
    plan = Plan.preset(query)
    with Context(0) as ctx:
        ctx.load(g)
        want = ctx.match(plan)
    dev = torch.device("cuda", 0)
    rp = torch.from_numpy(g.row_ptrs.view(np.int64)).to(dev)
    ci = torch.from_numpy(g.cols.view(np.int32)).to(dev)
    out = torch.full((1,), -1, dtype=torch.int64, device=dev)
    f = _noalloc(g2.lib())
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):  # the static scratch keeps the previous call's contents
        rc = f(rp.data_ptr(), ci.data_ptr(), g.n, g.m, C.addressof(plan.raw), out.data_ptr(), stream)
        assert rc == 0, g2.lib().g2_strerror(rc)
        torch.cuda.synchronize(dev)
        assert int(out.item()) == want


def test_noalloc_rejects_graphs_over_the_limit(g2):
    f = _noalloc(g2.lib())
    from g2aimd.context import Plan
    plan = Plan.preset(24)
    dummy = np.zeros(4, np.uint64)
    rc = f(dummy.ctypes.data, dummy.ctypes.data, (1 << 21) + 1, 0, C.addressof(plan.raw), dummy.ctypes.data, None)
    assert rc == -8  # G2_ERR_UNSUPPORTED, before any device work


def test_noalloc_overlapping_a_context_run_of_another_plan(g2):
    """The plan is a kernel argument: a no-alloc count of 4-cliques on one
    stream and a context's diamond count on another stream, enqueued back to
    back so that they may run at the same time, both give their own counts."""
    import torch

    from g2aimd.context import Context, Plan
    g = g2.Graph.rmat(13, 16, seed=23).degeneracy_recoded()
    k4, diamond = Plan.preset(24), Plan.preset(2)
    dev = torch.device("cuda", 0)
    rp = torch.from_numpy(g.row_ptrs.view(np.int64)).to(dev)
    ci = torch.from_numpy(g.cols.view(np.int32)).to(dev)
    f = _noalloc(g2.lib())
    with Context(0) as ctx:
        ctx.load(g)
        want_d = ctx.match(diamond)
        want_k4 = ctx.match(k4)
        ctx.set_plan(diamond)
        ctx.reserve()
        s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        out1 = torch.zeros(1, dtype=torch.int64, device=dev)
        out2 = torch.full((1,), -1, dtype=torch.int64, device=dev)
        torch.cuda.synchronize(dev)
        for _ in range(2):
            ctx.match_device(out1.data_ptr(), stream=s1.cuda_stream)
            rc = f(rp.data_ptr(), ci.data_ptr(), g.n, g.m, C.addressof(k4.raw), out2.data_ptr(), s2.cuda_stream)
            assert rc == 0, g2.lib().g2_strerror(rc)
            torch.cuda.synchronize(dev)
            assert int(out1.item()) == want_d
            assert int(out2.item()) == want_k4
