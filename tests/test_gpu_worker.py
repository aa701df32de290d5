"""g2_worker, the drop-in for the reference's `bk` / `run` binaries: same flags,
same result lines, in core (whole CSR per GPU) and out of core (-ooc 1: views
built by host threads, bins from the .vbmap or from -m)."""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORKER = os.path.join(ROOT, "g2-aimd_b200", "g2_worker")


def run_worker(*args):
    out = subprocess.run([WORKER, *map(str, args)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    return out.stdout


def cliques(stdout):
    return sum(int(x) for x in re.findall(r"^Total No\. of Cliques: (\d+)$", stdout, re.M))


def total_counts(stdout):
    return int(re.findall(r"^Total counts: (\d+)$", stdout, re.M)[-1])


def test_worker_bk_in_core_and_out_of_core(tmp_path, orc, c1_graph):
    g = c1_graph
    path = tmp_path / "c1.bin"
    g.write_bin(path)
    want = orc.mce(g, hist_len=64)["count"]
    assert cliques(run_worker("-dg", path, "-h", 2)) == want
    out = run_worker("-dg", path, "-h", 2, "-ooc", 1, "-pn", 3, "-m", 0.0001)  # 100 KB bins
    nbins = int(re.search(r"view bins: (\d+)", out).group(1))
    assert nbins > 1
    assert cliques(out) == want
    # bins from a .vbmap (the reference's file), round robin over one GPU
    bins = (np.arange(g.n) % 4).astype(np.uint32)
    g.write_vbmap(str(path) + ".2.hop.vbmap", 4, bins)
    out = run_worker("-dg", path, "-h", 2, "-ooc", 1, "-pn", 2)
    assert len(re.findall(r"^Total No\. of Cliques:", out, re.M)) == 4
    assert cliques(out) == want


@pytest.mark.parametrize("q", [0, 1, 24])
def test_worker_match_in_core_and_out_of_core(tmp_path, orc, g2, q):
    from g2aimd.context import Plan
    g = g2.Graph.rmat(10, 8, seed=8).degeneracy_recoded()
    path = tmp_path / "r10.bin"
    g.write_bin(path)
    want = orc.match(g, Plan.preset(q), threads=4)["count"]
    assert total_counts(run_worker("-dg", path, "-q", q)) == want
    out = run_worker("-dg", path, "-q", q, "-ooc", 1, "-pn", 4, "-m", 0.00001)  # 10 KB bins
    assert int(re.search(r"view bins: (\d+)", out).group(1)) > 1
    assert total_counts(out) == want
