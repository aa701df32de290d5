"""The device R-MAT generator (g2_gen_rmat_device) builds exactly the host
generator's CSR (g2_gen_rmat): same rows, planted cliques included, and the
device degeneracy recode of it equals the host recode."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,ef,planted", [(10, 8, 0), (15, 16, 0), (13, 16, 20), (17, 28, 0)])
def test_device_generator_equals_host(g2, scale, ef, planted):
    from g2aimd.context import Context
    kw = dict(planted=planted, pmin=20, pmax=60) if planted else {}
    want = g2.Graph.rmat(scale, ef, seed=9, **kw)
    with Context(0) as c:
        m = c.gen_rmat(scale, ef, seed=9, **kw)
        assert m == want.m
        got = c.copy_csr(m)
        assert np.array_equal(got.row_ptrs, want.row_ptrs)
        assert np.array_equal(got.cols, want.cols)
        perm, core = c.degeneracy_recode()
        rec = c.copy_csr(m)
        host = want.degeneracy_recoded()
        assert np.array_equal(rec.row_ptrs, host.row_ptrs) and np.array_equal(rec.cols, host.cols)
