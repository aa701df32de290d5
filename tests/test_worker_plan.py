"""g2_worker -plan 1 (no GPU): plans view bins for the query's view shape with
the -m budget, applies -ds/-dst/-dr, and writes the .vbmap that later runs
read, as the reference's offline view packing does."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORKER = os.path.join(ROOT, "g2-aimd_b200", "g2_worker")


def run(*args):
    out = subprocess.run([WORKER, *map(str, args)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    return out.stdout


def test_plan_writes_the_bins_of_g2_view_bins(g2, tmp_path):
    from g2aimd.context import Plan
    g = g2.Graph.rmat(10, 8, seed=8).degeneracy_recoded()
    path = tmp_path / "r10.bin"
    g.write_bin(path)
    # K4: the plan's hop names the file, the plan's view shape sizes the bins
    out = run("-dg", path, "-q", 24, "-plan", 1, "-m", 0.00001)
    nb = int(re.search(r"view bins: (\d+)", out).group(1))
    hop = Plan.preset(24).raw.hop
    vb = f"{path}.{hop}.hop.vbmap"
    assert os.path.exists(vb) and f"wrote {vb}" in out
    want_nb, want = g.view_bins(10000, **Plan.preset(24).view_shape())
    got_nb, got = g.read_vbmap(vb)
    assert nb == got_nb == want_nb > 1 and np.array_equal(got, want)
    # maximal cliques (-h names the file), split over 4 consumers and reordered
    out = run("-dg", path, "-h", 2, "-plan", 1, "-m", 0.0001, "-ds", 1, "-cn", 4, "-dr", 1)
    nb0, b0 = g.view_bins(100000, radius=1, row_radius=1, min_root_degree=1)
    want_nb, want = g.rebalance_bins(b0, nb0, devices=4, split_times=1, reorder=True)
    got_nb, got = g.read_vbmap(f"{path}.2.hop.vbmap")
    assert got_nb == want_nb == (nb0 // 4 + 1) * 4 and np.array_equal(got, want)


def py_shell_bins(core_new, nb):
    """kmeans/kcore.cpp:193-228 restated: each core shell (a run of ids in
    degeneracy order) in consecutive chunks of shell size // nb + 1 per bin."""
    out = np.zeros(core_new.size, np.uint32)
    i = 0
    while i < core_new.size:
        j = i
        while j < core_new.size and core_new[j] == core_new[i]:
            j += 1
        share = (j - i) // nb + 1
        out[i:j] = np.arange(j - i) // share
        i = j
    return out


def test_recode_writes_the_kcore_files(g2, tmp_path):
    g = g2.Graph.chung_lu(5000, 2.3, 8.0, seed=2)
    src = tmp_path / "cl.bin"
    dst = tmp_path / "cl_rec.bin"
    g.write_bin(src)
    out = run("-dg", src, "-recode", 1, "-o", dst, "-nb", 3)
    assert f"wrote {dst}" in out
    want = g.degeneracy_recoded()
    got = g2.Graph.read_bin(dst)
    assert np.array_equal(got.row_ptrs, want.row_ptrs) and np.array_equal(got.cols, want.cols)
    nb, bins = got.read_vbmap(f"{dst}.2.hop.vbmap")
    assert nb == 3 and np.array_equal(bins, py_shell_bins(want.core, 3))
    assert bins.max() == 2


SNAP = """# Directed graph (each unordered pair of nodes is saved once)
# FromNodeId\tToNodeId
5\t6
6\t7
7\t5
5\t6
9\t9
9\t10\textra column
12\t5

10\t11
"""


def py_snap(text, preprocess):
    """common/graph.h:268-358 and :720-804 restated."""
    edges = [tuple(int(x) for x in line.split()[:2]) for line in text.splitlines() if line[:1].isdigit()]
    lo = min(min(e) for e in edges)
    n = max(max(e) for e in edges) - lo + 1
    rows = [[] for _ in range(n)]
    for a, b in edges:
        rows[a - lo].append(b - lo)
        rows[b - lo].append(a - lo)
    rows = [sorted(r) for r in rows]
    if preprocess:
        rows = [sorted(set(v for v in r if v != u)) for u, r in enumerate(rows)]
        keep = [u for u in range(n) if rows[u]]
        new = {u: i for i, u in enumerate(keep)}
        rows = [[new[v] for v in rows[u]] for u in keep]
    rp = np.cumsum([0] + [len(r) for r in rows]).astype(np.uint64)
    ci = np.array([v for r in rows for v in r], np.uint32)
    return rp, ci


def test_read_snap_follows_the_reference(g2, tmp_path):
    path = tmp_path / "toy.txt"
    path.write_text(SNAP)
    for pre in (False, True):
        g = g2.Graph.read_snap(path, preprocess=pre)
        rp, ci = py_snap(SNAP, pre)
        assert np.array_equal(g.row_ptrs, rp) and np.array_equal(g.cols, ci), pre
    g = g2.Graph.read_snap(path)
    assert g.n == 7 and g.m == 12  # 8 never appears; 9-9 and the repeat of 5-6 are gone


def test_worker_prep_and_recode_read_snap_text(g2, tmp_path):
    path = tmp_path / "toy.txt"
    path.write_text(SNAP)
    out = run("-dg", path, "-prep", 1)
    assert f"wrote {tmp_path / 'toy.bin'}" in out
    got = g2.Graph.read_bin(tmp_path / "toy.bin")
    want = g2.Graph.read_snap(path)
    assert np.array_equal(got.row_ptrs, want.row_ptrs) and np.array_equal(got.cols, want.cols)
    run("-dg", path, "-recode", 1, "-o", tmp_path / "toy_rec.bin")
    rec = g2.Graph.read_bin(tmp_path / "toy_rec.bin")
    want = want.degeneracy_recoded()
    assert np.array_equal(rec.row_ptrs, want.row_ptrs) and np.array_equal(rec.cols, want.cols)


def test_read_snap_rejects_ids_beyond_32_bits(g2, tmp_path):
    path = tmp_path / "big.txt"
    path.write_text("1 4294967296\n")
    with pytest.raises(Exception):
        g2.Graph.read_snap(path)


def test_plan_threads_flag(g2, tmp_path, monkeypatch):
    """-t sets the planning threads: with -t 1 a large graph is planned in one
    range, as g2_view_bins plans it on one thread."""
    g = g2.Graph.chung_lu(1 << 17, 2.3, 10.0, seed=6).degeneracy_recoded()
    path = tmp_path / "cl17.bin"
    g.write_bin(path)
    budget_gb = (g.row_ptrs.nbytes + g.cols.nbytes) / 40 / 1e9
    run("-dg", path, "-h", 2, "-plan", 1, "-m", budget_gb, "-t", 1)
    monkeypatch.setenv("G2_HOST_THREADS", "1")
    want_nb, want = g.view_bins(int(budget_gb * 1e9), radius=1, row_radius=1, min_root_degree=1)
    got_nb, got = g.read_vbmap(f"{path}.2.hop.vbmap")
    assert got_nb == want_nb and np.array_equal(got, want)
