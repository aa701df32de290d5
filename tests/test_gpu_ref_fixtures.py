"""Counts at the benchmark configurations, pinned to the reference's own GPU build.

tests/golden/ref_gpu_counts.json holds what the reference's GPU programs
(app_gmatch `run`, app_BK `bk`, built from its sources by oracle/Makefile
`ref-gpu` and run on a B200 by oracle/ref_gpu_baseline.py) printed as
"Total counts:" / the sum of "Total No. of Cliques:" on graphs from this
library's seeded generators: C1 (ER 2000 + 5 K12), C2 (R-MAT s20 ef16:
triangles, 4-cliques), R-MAT s16 (4-cycles, diamonds, 4- and 5-cliques),
Chung-Lu graphs shaped like C3's stand-in and C4's members, and an R-MAT s13
with 20 planted cliques of 20-60 vertices.  A reference count is used only when
the run was trusted: exit code 0, no chunk retry (its GMatch double counts after
one), no host overflow, and record indices that fit in 32 bits.  The one count
it could not produce (5-cliques of R-MAT s20: its 4-clique level holds 6.8e10
entries) is checked instead against the plan walk (an independent device path)
and, per root, against the CPU oracle on a sample of roots.

Also at the headline size: per-root 4-clique counts on R-MAT s20 equal the
oracle's on 2,048 random roots plus the 16 heaviest.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = json.load(open(os.path.join(HERE, "golden", "ref_gpu_counts.json")))


def _graphs():
    import ref_gpu_baseline
    return {name: fn for name, _text, fn in ref_gpu_baseline.GRAPHS}


_cache = {}


def graph(g2, name):
    if name not in _cache:
        _cache.clear()  # one graph held at a time
        _cache[name] = _graphs()[name](g2.Graph).degeneracy_recoded()
    return _cache[name]


def _ref_count(r):
    return r["reference_gpu"]["cliques"] if r["job"] == "mce" else r["reference_gpu"]["counts"]


TRUSTED = [r for r in FIXTURE if r["reference_gpu"].get("trusted")]


def test_fixture_covers_the_configs():
    jobs = {(r["graph"], r["job"]) for r in TRUSTED}
    assert ("er2000_k12", "mce") in jobs            # C1
    assert {("rmat20", "q0"), ("rmat20", "q24")} <= jobs  # C2
    assert ("chunglu18", "mce") in jobs
    assert {("cl_5k", j) for j in ("mce", "q0", "q1", "q2")} <= jobs  # C4-shaped member
    assert len(TRUSTED) >= 20


@pytest.mark.parametrize("r", TRUSTED, ids=[f"{r['graph']}-{r['job']}" for r in TRUSTED])
def test_equals_reference_gpu_build(g2, ctx, r):
    from g2aimd.context import Plan
    g = graph(g2, r["graph"])
    assert (g.n, g.m) == (r["n"], r["m"])
    ctx.load(g)
    if r["job"] == "mce":
        ctx.load_core(g.core)
        count, _hist = ctx.mce(hist_len=256)
    else:
        count = ctx.match(Plan.preset(int(r["job"][1:])))
    assert count == _ref_count(r)


def _sample_roots(n, per_root, k_random, k_heavy, seed):
    rng = np.random.default_rng(seed)
    heavy = np.argsort(per_root, kind="stable")[-k_heavy:]
    rand = rng.choice(n, size=k_random, replace=False)
    return np.unique(np.concatenate([heavy, rand])).astype(np.uint32)


def test_rmat20_k4_per_root_equals_oracle(g2, orc, ctx):
    from g2aimd.context import Plan
    g = graph(g2, "rmat20")
    plan = Plan.preset(24)
    ctx.load(g)
    per = np.zeros(g.n, np.uint64)
    total = ctx.match(plan, root_counts=per)
    assert total == int(per.sum()) == 17038400522
    roots = _sample_roots(g.n, per, 2048, 16, 7)
    want = orc.match(g, plan, roots=roots, threads=os.cpu_count() or 1, per_root=True)["root_counts"]
    assert np.array_equal(per[roots], want)


def test_rmat20_k5_where_the_reference_cannot_count(g2, orc, ctx):
    from g2aimd.context import Plan
    r = [x for x in FIXTURE if (x["graph"], x["job"]) == ("rmat20", "q25")][0]
    assert not r["reference_gpu"]["trusted"]  # its record indices wrapped
    g = graph(g2, "rmat20")
    plan = Plan.preset(25)
    ctx.load(g)
    per = np.zeros(g.n, np.uint64)
    total = ctx.match(plan, root_counts=per)
    assert total == int(per.sum())
    # the generic plan walk (candidate lists + binary searches, hand-off) is
    # an independent device path: the same count for every root of a stride
    # sample (all roots through the walk take minutes)
    sample = np.arange(0, g.n, 512, dtype=np.uint32)
    per_walk = np.zeros(sample.size, np.uint64)
    assert ctx.match(plan, sources=sample, root_counts=per_walk, intersect_mode=1) == int(per[sample].sum())
    assert np.array_equal(per[sample], per_walk)
    # oracle on random roots and the 16 heaviest roots of at most 2e7 5-cliques
    # each (the heaviest hold ~1e9 each: minutes of CPU time per root)
    order = np.argsort(per, kind="stable")
    light = order[per[order] <= 20_000_000]
    rng = np.random.default_rng(11)
    roots = np.unique(np.concatenate([light[-16:], rng.choice(g.n, 1024, replace=False)])).astype(np.uint32)
    want = orc.match(g, plan, roots=roots, threads=os.cpu_count() or 1, per_root=True)["root_counts"]
    assert np.array_equal(per[roots], want)
