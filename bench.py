"""Benchmark: 4-clique matches/s on a seeded R-MAT scale-20 graph (edge factor
16, a=.57 b=c=.19, ids in degeneracy order) on one B200 per rank, with the
triangle count on the same graph and maximal-clique enumeration on a
power-law (Chung-Lu) graph reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one pass of the hot path over one batch: every root of the graph
expanded by the persistent plan-driven kernel for the 4-clique plan (preset 24),
task generation included: the learned cost model's features + MLP inference,
heavy-root splits, the device sort of the task list.  `value` is 4-clique
matches per second with the CSR resident in HBM, on the learned schedule whose
launch parameters the autotuner picked before the timed steps; the plain
schedule (heuristic order, one task per root) is timed the same way and
reported beside it.  `e2e` is the same metric through the host C ABI
(g2_load_csr + g2_load_core from pinned host memory, g2_match_run, count read
back) every step.  Maximal-clique enumeration is not
the headline on this graph: R-MAT graphs with edge factor 16 have a dense core
whose maximal-clique count grows ~10x per scale (measured up to scale 14), so
no implementation enumerates them at scale 20.  Under torchrun the ranks share
the graph and split its roots (longest-processing-time on degree x core); each
runs its shard and one exact all-reduce sums the counts ("scaling": "strong");
the timed region is bracketed by barriers and the max over ranks is reported.
`--impl reference` times the reference algorithm's CPU restatement (the
reference has only a GPU implementation) on the host cores, on the same graph
and every root.  Separate legs: --leg c5 (R-MAT scale 26, edge factor 28),
--leg c3 (maximal cliques of R-MAT with planted cliques), --leg mce, --leg view,
--leg view-host.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "g2-aimd_b200"))

import numpy as np  # noqa: E402

METRIC = "maximal cliques/s and 4-clique matches/s on 1 B200, learned vs plain schedule"
UNIT = "4-clique matches/s"
HIST = 256
K4 = 24


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=20, help="R-MAT scale (20 = the benchmark graph)")
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-sample-s", type=float, default=12.0, help="target seconds of CPU baseline work")
    ap.add_argument("--ref-budget-s", type=float, default=300.0,
                    help="reference arm: projected CPU seconds above which only 1/M of the roots is timed")
    ap.add_argument("--no-extras", action="store_true", help="skip triangle / MCE / e2e / CPU legs")
    ap.add_argument("--scratch-mb", type=int, default=4096, help="device scratch for the DFS slabs")
    ap.add_argument("--fixed", action="store_true",
                    help="skip the plain-schedule timing and the autotuner (profiling runs)")
    ap.add_argument("--leg", choices=["all", "mce", "view", "view-host", "c5", "c3", "c4", "walk"], default="all",
                    help="mce: only the maximal-clique workload (Chung-Lu 2^18), for profiling; "
                         "view: out-of-core runs over view bins against in-core runs; "
                         "view-host: the views' sizes and host build time alone (no GPU); "
                         "c4: the batch of 64 power-law graphs alone")
    ap.add_argument("--walk-query", type=int, default=1, help="preset plan of the walk leg (1: 4-cycles, 2: diamonds)")
    ap.add_argument("--view-split", type=int, default=2,
                    help="view leg: bin budget = CSR bytes / this")
    return ap.parse_args()


def ev_time(torch, stream, fn):
    """(result, device ms) of fn() between CUDA events on `stream`."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r = fn()
    e1.record(stream)
    e1.synchronize()
    return r, e0.elapsed_time(e1)


def wall_ms(torch, fn):
    """(result, ms) of a synchronous library call (device idle on both sides)."""
    torch.cuda.synchronize()
    t = time.perf_counter()
    r = fn()
    torch.cuda.synchronize()
    return r, 1000.0 * (time.perf_counter() - t)


def c5_leg(a, local, torch, stream, scale=26, ef=28, k5_stride=16384, mce_budget_ms=20000):
    """C5: R-MAT scale 26, edge factor 28, seed 1 (67 M vertices, 3.6 G directed
    entries, 15 GB CSR), built on the device (g2_gen_rmat_device) and put in
    degeneracy order on the device.  4-cliques and triangles over every root;
    4-cliques with the plain heuristic schedule and the learned one under the
    same launch parameters; 5-cliques over the roots v % k5_stride == 0 (all
    roots would take about an hour); maximal cliques with a device time budget
    (the count of maximal cliques explodes on R-MAT cores), reporting the roots
    that finished.  Device times between CUDA events on the run's stream."""
    import g2aimd  # noqa: F401
    from g2aimd.context import Context, CostModel, Plan
    models = os.path.join(ROOT, "g2-aimd_b200", "models")
    launch = {"warps_per_block": 4, "chunk": 1, "ctas_per_sm": 6}
    out = {"workload": f"rmat-s{scale}-ef{ef} (a=.57,b=c=.19, seed 1) degeneracy-ordered, built on the device"}
    # 48 GiB of slabs: the dense core's roots (|P0| up to ~4500) need 2.5 MB of rows each
    with Context(local, 48 << 30) as ctx:
        t0 = time.perf_counter()
        m = ctx.gen_rmat(scale, ef, seed=1)
        out["gen_s"] = round(time.perf_counter() - t0, 2)
        t0 = time.perf_counter()
        _perm, core = ctx.degeneracy_recode()
        out["recode_s"] = round(time.perf_counter() - t0, 2)
        out["graph"] = {"n": 1 << scale, "m": int(m), "degeneracy": int(core.max()),
                        "csr_bytes": int(8 * ((1 << scale) + 1) + 4 * m)}
        del _perm, core
        ctx.set_model(CostModel.load(os.path.join(models, "k4.npz")))
        sptr = stream.cuda_stream
        d_out = torch.zeros(1, dtype=torch.int64, device=torch.device("cuda", local))

        def count():
            stream.synchronize()
            return int(d_out[0].item())

        ctx.set_plan(Plan.preset(0))
        _, ms = ev_time(torch, stream, lambda: ctx.match_device(d_out.data_ptr(), stream=sptr, schedule="heuristic",
                                                               flags=1, **launch))
        out["triangle"] = {"count": count(), "ms": ms, "per_s": count() / (ms / 1000.0)}
        ctx.set_plan(Plan.preset(24))
        _, plain_ms = ev_time(torch, stream, lambda: ctx.match_device(
            d_out.data_ptr(), stream=sptr, schedule="given", flags=1, **launch))
        k4 = count()
        _, heur_ms = ev_time(torch, stream, lambda: ctx.match_device(
            d_out.data_ptr(), stream=sptr, schedule="heuristic", flags=1, **launch))
        assert count() == k4
        _, learned_ms = ev_time(torch, stream, lambda: ctx.match_device(
            d_out.data_ptr(), stream=sptr, schedule="learned", flags=1 | 8, **launch))
        assert count() == k4, (count(), k4)
        out["k4"] = {"count": k4, "plain_kcore_order_ms": plain_ms, "plain_heuristic_ms": heur_ms,
                     "learned_ms": learned_ms, "learned_vs_plain": plain_ms / learned_ms,
                     "learned_vs_degree_core_heuristic": heur_ms / learned_ms, "per_s": k4 / (learned_ms / 1000.0),
                     "launch": launch, "note": "plain = the reference's kcore root order; no heavy-root splits, "
                                               "same launch parameters"}
        roots = np.arange(0, 1 << scale, k5_stride, dtype=np.uint32)
        d_roots = torch.from_numpy(roots.view(np.int32)).to(d_out.device)
        ctx.set_plan(Plan.preset(25))
        _, ms = ev_time(torch, stream, lambda: ctx.match_device(
            d_out.data_ptr(), d_roots.data_ptr(), roots.size, stream=sptr, schedule="heuristic", flags=1, **launch))
        k5 = count()
        out["k5_sample"] = {"roots": f"v % {k5_stride} == 0 ({roots.size} roots)", "count": k5, "ms": ms,
                            "per_s": k5 / (ms / 1000.0), "scaled_total_estimate": k5 * k5_stride}
        # maximal cliques: light roots first (degeneracy order), a device time budget
        ctx.set_model(CostModel.load(os.path.join(models, "mce.npz")))
        t0 = time.perf_counter()
        c, _h, rn = ctx.mce(hist_len=4096, root_nodes=True, deadline_ms=mce_budget_ms, flags=1)
        wall = time.perf_counter() - t0
        done = int(np.count_nonzero(rn))
        out["mce_budgeted"] = {"budget_ms": mce_budget_ms, "wall_s": round(wall, 2), "expired": bool(ctx.expired),
                               "roots_finished": done, "maximal_cliques_of_finished_roots": int(c),
                               "search_tree_nodes": int(rn.sum()),
                               "per_s": c / wall if wall else None,
                               "order": "root ids in degeneracy order (light roots first), one warp per root"}
    return out


def c3_leg(a, local, torch, stream, reps=3, budget_ms=30000):
    """C3 in the form that completes: maximal cliques of R-MAT ef16 (seed 1)
    grow ~10x per scale, so scale 24 + 200 planted cliques cannot be enumerated
    by any implementation.  Recorded here: (1) the growth, full counts with
    hand-off at scales 10-15 and a time-budgeted run at 16 (roots finished);
    (2) C3's question, learned vs plain schedule (same launch, same hand-off),
    on R-MAT s14 and s15 ef16 with 200 planted cliques of 20-60 vertices
    planted exactly as C3 plants them (g2_gen_rmat's planted cliques)."""
    from g2aimd.context import Context, CostModel, Plan  # noqa: F401
    models = os.path.join(ROOT, "g2-aimd_b200", "models")
    out = {"growth": [], "planted": []}
    with Context(local) as ctx:
        ctx.set_model(CostModel.load(os.path.join(models, "mce.npz")))
        for sc in range(10, 17):
            m = ctx.gen_rmat(sc, 16, seed=1)
            ctx.degeneracy_recode()
            rec = {"scale": sc, "m": int(m)}
            if sc <= 15:
                ctx.mce(hist_len=256, flags=1)  # warm-up (buffers)
                (c, _h), ms = wall_ms(torch, lambda: ctx.mce(hist_len=256, flags=1))
                rec.update({"maximal_cliques": int(c), "ms": ms})
            else:
                t0 = time.perf_counter()
                c, _h, rn = ctx.mce(hist_len=4096, root_nodes=True, flags=1, deadline_ms=budget_ms)
                rec.update({"budget_ms": budget_ms, "expired": bool(ctx.expired), "wall_s":
                            round(time.perf_counter() - t0, 2), "roots_finished": int(np.count_nonzero(rn)),
                            "maximal_cliques_of_finished_roots": int(c)})
            out["growth"].append(rec)
        for sc in (14, 15):
            m = ctx.gen_rmat(sc, 16, planted=200, pmin=20, pmax=60, seed=1)
            ctx.degeneracy_recode()
            rec = {"graph": f"rmat-s{sc}-ef16 + 200 planted cliques of 20-60 vertices (seed 1)", "m": int(m)}
            res = {}
            for sched in ("given", "heuristic", "learned"):
                run = lambda sched=sched: ctx.mce(hist_len=256, schedule=sched, flags=1)  # noqa: E731
                run()
                times = []
                for _ in range(reps):
                    (c, h), ms = wall_ms(torch, run)
                    times.append(ms)
                res[sched] = (int(c), h, float(np.median(times)))
            for sched in ("given", "heuristic"):
                assert res[sched][0] == res["learned"][0]
                assert np.array_equal(res[sched][1], res["learned"][1])
            rec.update({"maximal_cliques": res["learned"][0], "plain_kcore_order_ms": res["given"][2],
                        "plain_heuristic_ms": res["heuristic"][2], "learned_ms": res["learned"][2],
                        "learned_vs_plain": res["given"][2] / res["learned"][2],
                        "learned_vs_degree_core_heuristic": res["heuristic"][2] / res["learned"][2],
                        "largest_clique": int(np.flatnonzero(res["learned"][1])[-1]),
                        "note": "same hand-off and launch parameters; histograms equal"})
            out["planted"].append(rec)
    return out


def run_c3_leg(a):
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    print(json.dumps(c3_leg(a, 0, torch, stream)), flush=True)


def run_c5_leg(a):
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    print(json.dumps(c5_leg(a, 0, torch, stream)), flush=True)


def run_c4_leg(a):
    import torch

    from g2aimd.context import Context, CostModel, Plan
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    models = os.path.join(ROOT, "g2-aimd_b200", "models")
    print(json.dumps(c4_leg(Context, CostModel, Plan, models, 0, a.seed, torch, stream)), flush=True)


def run_walk_leg(a):
    """Plan walks alone (for profiling): 4-cycles (preset 1; --walk-query picks
    another preset) on a Chung-Lu graph shaped like the larger C4 members
    (n = 2e5, gamma 2.2, average degree 20), heuristic order with hand-off, W
    warm-up and K timed runs; one JSON line."""
    import torch

    import g2aimd
    from g2aimd.context import Context, Plan
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    g = g2aimd.Graph.chung_lu(200000, 2.2, 20.0, seed=1).degeneracy_recoded()
    out = torch.zeros(1, dtype=torch.int64, device=dev)
    with Context(0) as ctx:
        ctx.load(g)
        ctx.load_core(g.core)
        ctx.set_plan(Plan.preset(a.walk_query))
        run = lambda: ctx.match_device(out.data_ptr(), stream=stream.cuda_stream, schedule="heuristic", flags=1)  # noqa
        for _ in range(a.warmup):
            run()
        times = [ev_time(torch, stream, run)[1] for _ in range(a.steps)]
        name = {1: "4-cycles", 2: "diamonds"}.get(a.walk_query, f"preset {a.walk_query}")
        print(json.dumps({"workload": f"{name}, chung-lu n=2e5 gamma 2.2 avg degree 20", "count": int(out[0].item()),
                          "ms": times}), flush=True)


def run_mce_leg(a):
    """Maximal cliques on the Chung-Lu graph (n = 2^18, gamma 2.3, average degree
    16) with hand-off, W warm-up and K timed runs; one JSON line (device times)."""
    import torch

    import g2aimd
    from g2aimd.context import Context
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = g2aimd.Graph.chung_lu(1 << 18, 2.3, 16.0, seed=a.seed).degeneracy_recoded()
    with Context(0, a.scratch_mb << 20) as ctx:
        ctx.load(g)
        ctx.reserve()
        for _ in range(a.warmup):
            c, _h = ctx.mce(schedule="heuristic", flags=1)
        times = []
        for _ in range(a.steps):
            c, _h = ctx.mce(schedule="heuristic", flags=1)
            times.append(ctx.pass_times()[0])
        print(json.dumps({"workload": "mce chung-lu n=2^18 gamma 2.3 avg degree 16", "maximal_cliques": int(c),
                          "kernel_ms": times, "records": ctx.spill_stats()[0]}), flush=True)


def view_legs(a, g, steps, warmup):
    """Out-of-core enumeration (g2_view_match / g2_view_mce: CSR in pinned host
    memory, views built by host threads, uploads overlapping the runs) against
    the in-core path (upload the whole CSR, then run) on the same host graph,
    both timed end to end on the host: 4-cliques on `g` and maximal cliques on
    the Chung-Lu graph (n = 2^18, gamma 2.3, average degree 16)."""
    import torch

    import g2aimd
    from g2aimd.context import Context, Plan
    producers = min(16, os.cpu_count() or 1)
    launch = {"warps_per_block": 8, "chunk": 1, "ctas_per_sm": 6}
    out = {"workload": "out-of-core view bins vs in-core, host CSR in pinned memory, bins of CSR bytes / "
                       f"{a.view_split}", "producers": producers}

    def pinned(g):
        prp = torch.from_numpy(g.row_ptrs.view(np.int64)).pin_memory()
        pci = torch.from_numpy(g.cols.view(np.int32)).pin_memory()
        return g2aimd.Graph(prp.numpy().view(np.uint64), pci.numpy().view(np.uint32)), (prp, pci)

    def leg(name, g, shape, view_fn, core_fn, device_fn=None):
        csr = g.row_ptrs.nbytes + g.cols.nbytes
        budget = csr // a.view_split
        t0 = time.perf_counter()
        nb, bins = g.view_bins(budget, **shape)
        bin_s = time.perf_counter() - t0
        pg, keep = pinned(g)
        with Context(0, a.scratch_mb << 20) as ctx:
            for _ in range(warmup):
                c_view, st = view_fn(ctx, pg, bins, nb)
            vt = []
            for _ in range(steps):
                t0 = time.perf_counter()
                c_view, st = view_fn(ctx, pg, bins, nb)
                vt.append((time.perf_counter() - t0) * 1e3)
            dvt, c_dev, st_dev = [], None, None
            if device_fn is not None:  # the same views built by the GPU (G2_VIEW_DEVICE)
                for _ in range(warmup):
                    c_dev, st_dev = device_fn(ctx, pg, bins, nb)
                for _ in range(steps):
                    t0 = time.perf_counter()
                    c_dev, st_dev = device_fn(ctx, pg, bins, nb)
                    dvt.append((time.perf_counter() - t0) * 1e3)
            for _ in range(warmup):
                ctx.load(pg)
                c_core = core_fn(ctx)
            ct = []
            for _ in range(steps):
                t0 = time.perf_counter()
                ctx.load(pg)
                c_core = core_fn(ctx)
                ct.append((time.perf_counter() - t0) * 1e3)
        assert c_view == c_core, (name, c_view, c_core)
        assert c_dev is None or c_dev == c_core, (name, c_dev, c_core)
        del keep
        out[name] = {"graph": {"n": g.n, "m": g.m}, "shape": shape, "csr_bytes": int(csr),
                     "bin_budget_bytes": int(budget), "bins": nb, "bin_plan_s": round(bin_s, 3),
                     "count": int(c_view), "view_ms": float(np.mean(vt)), "in_core_ms": float(np.mean(ct)),
                     "view_vs_in_core": float(np.mean(ct)) / float(np.mean(vt)), "stats": st}
        if dvt:
            out[name].update({"device_built_view_ms": float(np.mean(dvt)),
                              "device_built_vs_in_core": float(np.mean(ct)) / float(np.mean(dvt)),
                              "device_built_stats": st_dev})

    k4 = Plan.preset(K4)
    leg(f"k4_rmat_s{a.scale}", g, k4.view_shape(),
        lambda ctx, pg, bins, nb: (lambda c, _pb, st: (c, st))(
            *ctx.view_match(pg, bins, k4, nbins=nb, producers=producers, schedule="heuristic", **launch)),
        lambda ctx: ctx.match(k4, schedule="heuristic", **launch),
        lambda ctx, pg, bins, nb: (lambda c, _pb, st: (c, st))(
            *ctx.view_match(pg, bins, k4, nbins=nb, device=True, schedule="heuristic", **launch)))
    cl = g2aimd.Graph.chung_lu(1 << 18, 2.3, 16.0, seed=a.seed).degeneracy_recoded()
    leg("mce_chung_lu_2^18", cl, {"radius": 1, "row_radius": 1, "min_root_degree": 1, "upper": False},
        lambda ctx, pg, bins, nb: (lambda c, _h, _pb, st: (c, st))(
            *ctx.view_mce(pg, bins, nbins=nb, hist_len=HIST, producers=producers, schedule="heuristic")),
        lambda ctx: ctx.mce(hist_len=HIST, schedule="heuristic")[0],
        lambda ctx, pg, bins, nb: (lambda c, _h, _pb, st: (c, st))(
            *ctx.view_mce(pg, bins, nbins=nb, hist_len=HIST, device=True, schedule="heuristic")))
    return out


def run_view_host_leg(a):
    """Bins and view sizes of the view legs' workloads, built on the host through
    g2_view_bins / g2_view_materialize (one thread), for each view shape the
    query allows (full balls and rows, upper balls, upper balls + forward rows)."""
    import g2aimd
    from g2aimd.context import Plan
    g, _ = make_graph(a.scale, a.edge_factor, a.seed)
    cl = g2aimd.Graph.chung_lu(1 << 18, 2.3, 16.0, seed=a.seed).degeneracy_recoded()
    k4 = Plan.preset(K4).view_shape()
    mce = {"radius": 1, "row_radius": 1, "min_root_degree": 1, "upper": False, "forward": False}
    out = {"workload": f"view bins of CSR bytes / {a.view_split}, built on the host (no GPU); ego rows on "
                       "the bins planned without them"}
    cases = [(f"k4_rmat_s{a.scale}", g, dict(k4, upper=False, forward=False)),
             (f"k4_rmat_s{a.scale}", g, dict(k4, forward=False)), (f"k4_rmat_s{a.scale}", g, k4),
             (f"k4_rmat_s{a.scale}", g, dict(k4, ego=True)),
             ("mce_chung_lu_2^18", cl, mce), ("mce_chung_lu_2^18", cl, dict(mce, ego=True))]
    for name, gr, shape in cases:
        budget = (gr.row_ptrs.nbytes + gr.cols.nbytes) // a.view_split
        t0 = time.perf_counter()
        nb, bins = gr.view_bins(budget, **shape)
        plan_s = time.perf_counter() - t0
        order = np.argsort(bins, kind="stable")
        cuts = np.searchsorted(bins[order], np.arange(nb + 1))
        vn = vm = 0
        t0 = time.perf_counter()
        for b in range(nb):
            v, _src, _ids = gr.view(order[cuts[b]:cuts[b + 1]].astype(np.uint32), **shape)
            vn += v.n
            vm += v.m
        key = name + ("/forward" if shape["forward"] else "/upper" if shape["upper"] else "/full") + \
            ("+ego" if shape.get("ego") else "")
        out[key] = {"bins": nb, "plan_s": round(plan_s, 2), "view_vertices": int(vn), "view_entries": int(vm),
                    "entries_vs_m": round(vm / gr.m, 3), "build_s": round(time.perf_counter() - t0, 2)}
    print(json.dumps(out), flush=True)


def run_view_leg(a):
    """The view legs alone (one JSON line)."""
    import torch
    torch.cuda.set_device(torch.device("cuda", 0))
    g, _ = make_graph(a.scale, a.edge_factor, a.seed)
    print(json.dumps(view_legs(a, g, a.steps, a.warmup)), flush=True)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_graph(scale, ef, seed):
    import g2aimd
    t = time.perf_counter()
    g = g2aimd.Graph.rmat(scale, ef, 0.57, 0.19, 0.19, seed=seed).degeneracy_recoded()
    return g, time.perf_counter() - t


class Clocks:
    """nvidia-smi samples (every 200 ms) during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def c4_work_estimate(g):
    """Host estimate of the plan walk's work for 4-vertex patterns rooted at a
    vertex's forward neighbourhood: sum over roots v of |N+(v)| / 2 x the degree
    sum of N+(v) (used to keep the 4-cycle / diamond legs bounded)."""
    rp = g.row_ptrs.astype(np.int64)
    deg = np.diff(rp)
    src = np.repeat(np.arange(g.n), deg)
    dst = g.cols.astype(np.int64)
    fw = dst > src
    pf = np.bincount(src[fw], minlength=g.n)
    s1 = np.bincount(src[fw], weights=deg[dst[fw]], minlength=g.n)
    return float((s1 * pf).sum() / 2)


def c4_leg(Context, CostModel, Plan, models, local, seed, torch, stream, budget_ms=1000):
    """64 Chung-Lu graphs (n log-uniform in [1e3, 1e6], exponent in [2.1, 2.8],
    average degree in [8, 40]): triangles over all of them, maximal cliques over
    the ones of degeneracy <= 160 (the densest cores hold 5e9 to over 3e10
    maximal cliques each), diamonds over all of them, 4-cycles over the ones
    whose estimated walk is at most 1e10; each job is one launch over the batch
    (disjoint union), compared with one run per graph.  The members left out of
    a job then run it alone with a device time budget (budget_ms), reporting the
    roots that finished and their exact counts."""
    from g2aimd.graph import chung_lu_batch
    t0 = time.perf_counter()
    gs = chung_lu_batch(count=64, seed=seed)
    gen_s = time.perf_counter() - t0
    est = [c4_work_estimate(g) for g in gs]
    light = [g for g, e in zip(gs, est) if e <= 1e10]
    mce_set = [g for g in gs if int(g.core.max()) <= 160]

    def ev_ms(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), r

    jobs = [("triangle", 0, gs), ("diamond", 2, gs), ("mce", None, mce_set), ("4-cycle", 1, light)]
    out = {"graphs": len(gs), "vertices": int(sum(g.n for g in gs)), "directed_edges": int(sum(g.m for g in gs)),
           "generation_s": round(gen_s, 1), "mce_graphs": len(mce_set), "mce_rule": "degeneracy <= 160",
           "light_graphs": len(light), "light_rule": "4-cycles: estimated 4-vertex walk <= 1e10; diamonds: all"}
    with Context(local) as bc:
        bc.set_model(CostModel.load(os.path.join(models, "mce.npz")))
        loaded = None
        for name, q, members in jobs:
            if loaded is not members:
                bc.batch_load(members)
                bc.reserve()
                loaded = members
            run = (lambda: bc.batch_mce(schedule="learned")[0]) if q is None else \
                (lambda q=q: bc.batch_match(Plan.preset(q), schedule="heuristic"))
            run()
            ms, counts = min((ev_ms(run) for _ in range(3)), key=lambda x: x[0])
            out[name] = {"batched_ms": ms, "total": int(np.sum(counts)), "graphs": len(members)}
        # one graph at a time: a load, then the same job, device time of the jobs only
        for name, q, members in jobs:
            tot, cnt = 0.0, 0
            for g in members:
                bc.load(g)
                if q is None:
                    bc.load_core(g.core)
                run = (lambda: bc.mce(schedule="learned")[0]) if q is None else \
                    (lambda q=q: bc.match(Plan.preset(q), schedule="heuristic"))
                run()
                ms, c = ev_ms(run)
                tot += ms
                cnt += int(c)
            assert cnt == out[name]["total"], (name, cnt, out[name]["total"])
            out[name]["per_graph_loop_ms"] = tot
            out[name]["batched_vs_loop"] = tot / out[name]["batched_ms"]
        # the members left out above, each job with a device time budget: the
        # roots that finished and their exact counts (MCE: root_nodes > 0;
        # matches: root_cost > 0)
        heavy = []
        for gi, g in enumerate(gs):
            jobs_g = ([("mce", None)] if g not in mce_set else []) + ([("4-cycle", 1)] if g not in light else [])
            if not jobs_g:
                continue
            bc.load(g)
            bc.load_core(g.core)
            rec = {"graph": gi, "n": g.n, "m": g.m, "degeneracy": int(g.core.max()), "walk_estimate": est[gi]}
            for name, q in jobs_g:
                t0 = time.perf_counter()
                if q is None:
                    c, _h, rn = bc.mce(hist_len=4096, root_nodes=True, flags=1, deadline_ms=budget_ms)
                    done = int(np.count_nonzero(rn))
                else:
                    cost = np.zeros(g.n, np.uint64)
                    c = bc.match(Plan.preset(q), root_cost=cost, schedule="heuristic", flags=1,
                                 deadline_ms=budget_ms)
                    done = int(np.count_nonzero(cost))
                rec[name] = {"count_of_finished_roots": int(c), "roots_finished": done, "complete": not bc.expired,
                             "wall_s": round(time.perf_counter() - t0, 2)}
            heavy.append(rec)
        out["left_out_members_budgeted"] = {"budget_ms": budget_ms, "graphs": heavy}
    return out


def headline_profile():
    """Figures of the headline kernel's ncu capture committed under profiles/
    (R-MAT s20 ef16 seed 1, 4-cliques): DRAM bytes per launch and warp
    instructions per launch."""
    path = os.path.join(ROOT, "profiles", "match_kernel_k4_rmat_s20.md")
    out = {"file": "profiles/match_kernel_k4_rmat_s20.md"}
    try:
        text = open(path).read()
    except OSError:
        return out
    import re
    m = re.search(r"DRAM traffic per launch[^|]*\|\s*([0-9.,]+) MB", text)
    if m:
        out["traffic"] = float(m.group(1).replace(",", "")) * 1e6
    m = re.search(r"smsp__inst_executed\.sum\s*\|\s*([0-9.,]+) G", text)
    if m:
        out["inst"] = float(m.group(1).replace(",", "")) * 1e9
    return out


def cpu_stride_sample(g, stride, threads):
    """4-cliques of the roots v % stride == 0 by the CPU restatement of the
    reference algorithm (oracle/g2_oracle.c), heaviest roots first."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    from g2aimd.context import Plan
    ids = np.arange(g.n - 1, -1, -1, dtype=np.uint32)
    roots = ids[ids % stride == 0]
    orc.match(g, Plan.preset(K4), roots=roots[:64], threads=threads)  # thread pool start
    t = time.perf_counter()
    cnt = orc.match(g, Plan.preset(K4), roots=roots, threads=threads)["count"]
    spent = time.perf_counter() - t
    return {"value": cnt / spent, "roots": int(roots.size), "seconds": spent, "count": cnt}


def cpu_sample(g, target_s, threads, what="k4"):
    """The CPU restatement of the reference algorithm (oracle/g2_oracle.c) on a
    bounded random sample of roots, grown until it takes about target_s.
    Returns matches (or maximal cliques) per second on that sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    from g2aimd.context import Plan
    plan = Plan.preset(K4) if what == "k4" else None
    rng = np.random.default_rng(12345)
    perm = rng.permutation(g.n).astype(np.uint32)
    size, spent, cnt = 4096, 0.0, 0
    while True:
        roots = perm[:size]
        t = time.perf_counter()
        if plan is not None:
            cnt = orc.match(g, plan, roots=roots, threads=threads)["count"]
        else:
            cnt = orc.mce(g, roots=roots, threads=threads, hist_len=HIST)["count"]
        spent = time.perf_counter() - t
        if spent >= target_s or size >= g.n:
            break
        size = min(g.n, int(size * max(2.0, min(8.0, target_s / max(spent, 1e-3)))))
    return {"value": cnt / spent, "roots": int(size), "seconds": spent, "count": cnt}


def bench_config(a, n, m, world):
    """The `config` of both arms' lines (identical for the same workload)."""
    return {"workload": f"rmat-s{a.scale}-ef{a.edge_factor} (a=.57,b=c=.19, seed {a.seed}) degeneracy-ordered: "
                        "4-clique count (preset 24 plan) over all roots",
            "graph": {"n": int(n), "m": int(m), "seed": a.seed},
            "parallelism": f"dp{world}: the roots of one graph split over ranks (LPT on degree x core), "
                           "one all-reduce of the count"}


def run_reference(a):
    """The reference algorithm on the host cores, on the same graph and roots.

    The reference has only a GPU implementation; its CPU restatement
    (oracle/g2_oracle.c: plan-driven enumeration with the reference planner's
    plan, all host threads) stands in for it.  The graph is built by the oracle
    itself (the seeded generator and the kcore-tool recode restated in C), so
    nothing of the library is loaded.  Timed step i counts the 4-cliques rooted
    at the vertices v with v % (K * M) == i (heaviest roots first), so the K
    timed steps together cover every root exactly once when M = 1: the line's
    value is then the whole graph's count over the whole run's time, the same
    workload as the GPU arm's.  M > 1 only if the warm-up steps (roots
    v % 512 == j) project more than --ref-budget-s of CPU time for all roots;
    the covered fraction 1/M is then reported."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    import math
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    t0 = time.perf_counter()
    g = orc.degeneracy_recoded(orc.gen_rmat(a.scale, a.edge_factor, 0.57, 0.19, 0.19, seed=a.seed))
    build_s = time.perf_counter() - t0
    plan = orc.PresetPlan(K4)
    threads = os.cpu_count() or 1
    ids = np.arange(g.n - 1, -1, -1, dtype=np.uint32)  # late (dense-core) roots first
    spent, frac = 0.0, 0.0
    for j in range(a.warmup):
        roots = ids[ids % 512 == j]
        t = time.perf_counter()
        orc.match(g, plan, roots=roots, threads=threads)
        if j or a.warmup == 1:  # the first call also starts the thread pool
            spent += time.perf_counter() - t
            frac += roots.size / g.n
    projected = spent / frac if frac else 0.0
    M = max(1, math.ceil(projected / a.ref_budget_s)) if projected else 1
    stride = a.steps * M
    counts, times = [], []
    for i in range(a.steps):
        roots = ids[ids % stride == i]
        t = time.perf_counter()
        counts.append(orc.match(g, plan, roots=roots, threads=threads)["count"])
        times.append(time.perf_counter() - t)
    total, secs = int(sum(counts)), float(sum(times))
    v = total / secs
    cover = "every root once over the timed steps" if M == 1 else f"1/{M} of the roots (v % {stride} < {a.steps})"
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000.0 * secs / a.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": bench_config(a, g.n, g.m, world),
        "count": total, "roots_covered": int(np.count_nonzero((ids % stride) < a.steps)),
        "graph_build_s": round(build_s, 2), "projected_full_s": round(projected, 1),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{cover}: step i takes the roots v % {stride} == i, plan-driven enumeration "
                                   "with the reference planner's plan (oracle/g2_oracle.c, all host threads; "
                                   "graph built by the oracle)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def e2e_leg(a, g, roots, tuned, total, dev, local, world, torch, models, dist):
    """The headline metric end to end through the host C ABI: every step loads
    the CSR and the core numbers from pinned host memory (g2_load_csr,
    g2_load_core), runs g2_match_run over this rank's roots and reads the count
    back; wall time per step, the max over ranks."""
    import g2aimd
    from g2aimd.context import Context, CostModel, Plan
    prp = torch.from_numpy(g.row_ptrs.view(np.int64)).pin_memory()
    pci = torch.from_numpy(g.cols.view(np.int32)).pin_memory()
    pcore = torch.from_numpy(g.core.view(np.int32)).pin_memory()
    pg = g2aimd.Graph(prp.numpy().view(np.uint64), pci.numpy().view(np.uint32))
    core_h = pcore.numpy().view(np.uint32)
    e2c = Context(local)
    e2c.set_model(CostModel.load(os.path.join(models, "k4.npz")))
    plan = Plan.preset(K4)

    def e2e_step():
        e2c.load(pg)
        e2c.load_core(core_h)
        return e2c.match(plan, sources=roots, schedule="learned", **dict(tuned, flags=tuned["flags"] & ~1))

    for _ in range(a.warmup):
        e2e_step()
    torch.cuda.synchronize(dev)
    if dist:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        c2 = e2e_step()
    e2e_s = (time.perf_counter() - t0) / a.steps
    if dist:
        from g2aimd.shard import allreduce_counts
        mx = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(mx[0])
        c2, _ = allreduce_counts(c2, device=dev)
    assert c2 == total, (c2, total)
    e2c.close()
    return {"value": total / e2e_s, "unit": UNIT,
            "h2d_bytes_per_step": int(g.row_ptrs.nbytes + g.cols.nbytes + g.core.nbytes),
            "d2h_bytes_per_step": 8}


def run_ours(a):
    import ctypes

    import torch

    import g2aimd
    from g2aimd.autotune import DEFAULT_SPACE, tune
    # flags: heavy-root splits on (1) or off (1 | 8), L2 persistence window (| 32)
    LEARNED_SPACE = dict({"flags": [1, 1 | 8, 1 | 8 | 32, 1 | 32]}, **DEFAULT_SPACE)
    # MCE: hand-off check interval and queue chunk
    FLAG_NO_SPILL = 16
    MCE_SPACE = {"spill_kcycles": [5, 20, 100], "chunk": [1, 2], "warps_per_block": [4, 8]}
    from g2aimd.context import Context, CostModel, Plan
    world, rank, local = dist_env()
    dist = world > 1
    if dist:
        import datetime

        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    # a created stream for everything timed: stream attributes (the L2 window
    # option) apply to created streams, not to the legacy default stream
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    L = g2aimd.lib()
    models = os.path.join(ROOT, "g2-aimd_b200", "models")
    g, gen_s = make_graph(a.scale, a.edge_factor, a.seed)
    # ranks share the graph and split its roots (LPT on degree x core, the plain
    # heuristic's cost); one exact all-reduce of the count ends a run
    roots = None
    if dist:
        from g2aimd.shard import allreduce_counts, shard
        cost = (g.degrees().astype(np.float64) + 1.0) * (g.core.astype(np.float64) + 1.0)
        roots = shard(g.n, world, rank, cost)
        d_src = torch.from_numpy(roots.view(np.int32)).to(dev)
    ctx = Context(local, a.scratch_mb << 20)
    rp = torch.from_numpy(g.row_ptrs.view(np.int64)).to(dev)
    ci = torch.from_numpy(g.cols.view(np.int32)).to(dev)
    ctx.load_device(rp.data_ptr(), ci.data_ptr(), g.n, g.m)
    ctx.load_core(g.core)
    ctx.set_model(CostModel.load(os.path.join(models, "k4.npz")))
    out = torch.zeros(1 + HIST, dtype=torch.int64, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)  # > L2 (126 MB)
    sptr = stream.cuda_stream
    cur = {"ctx": ctx}

    def timed(fn, steps, warm):
        """Device time of each step (CUDA events on the launching stream, L2
        flushed before each step) and of the main enumeration pass."""
        for _ in range(warm):
            fn()
        torch.cuda.synchronize(dev)
        ms, pass_ms = [], []
        for _ in range(steps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            f = ctypes.c_float()
            if L.g2_pass_time_ms(cur["ctx"].handle, 0, ctypes.byref(f)) == 0:
                pass_ms.append(f.value)
        return ms, pass_ms

    def work_of(c):
        wb = ctypes.c_uint64()
        g2aimd._lib.check(L.g2_last_work_bytes(c.handle, ctypes.byref(wb)), "work")
        return wb.value

    def count():
        torch.cuda.synchronize(dev)
        return int(out[0].item())

    # ---- 4-clique count over every root (preset 24 plan)
    ctx.set_plan(Plan.preset(K4))
    if dist:
        run = lambda **kw: ctx.match_device(out.data_ptr(), d_src.data_ptr(), roots.size, stream=sptr, **kw)  # noqa
    else:
        run = lambda **kw: ctx.match_device(out.data_ptr(), stream=sptr, **kw)  # noqa: E731
    run(schedule="heuristic", flags=2)  # work-model build (schedule-independent), untimed
    work_bytes = work_of(ctx)
    k4 = count()
    if a.fixed:
        # the configuration the autotuner settles on for this workload (no splits, 4 warps per CTA)
        plain_ms, tuned, tlog = [float("nan")], {"flags": 1 | 8, "granularity": 64, "warps_per_block": 4,
                                                 "chunk": 1, "ctas_per_sm": 6}, []
    else:
        # plain schedule: heuristic order, one task per root (no model, no splits)
        plain_ms, _ = timed(lambda: run(schedule="heuristic", flags=1), a.steps, a.warmup)
        # learned schedule: autotuned launch/split parameters (untimed search)
        tuned, _, tlog = tune(lambda **kw: run(schedule="learned", **kw),
                              {"flags": 1, "granularity": 4, "warps_per_block": 8, "chunk": 4}, LEARNED_SPACE)
    step = lambda: run(schedule="learned", **tuned)  # noqa: E731
    step()
    assert count() == k4
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    with Clocks(local) as clk:
        ms, pass_ms = timed(step, a.steps, a.warmup)
    launches_per_step = ctx.launches()
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    step_ms = float(np.sum(ms)) / a.steps
    if dist:
        mx = torch.tensor([step_ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        step_ms_all = float(mx[0])
        total, _ = allreduce_counts(k4, device=dev)  # this rank's shard count -> the graph's
    else:
        step_ms_all, total = step_ms, k4
    value = total / (step_ms_all / 1000.0)
    kern_ms = float(np.mean(pass_ms)) if pass_ms else None
    # the plain heuristic schedule with everything else the learned run has
    # (launch parameters, hand-off, heavy-root splits iff the learned run splits):
    # the two differ in the schedule alone
    plain_flags = tuned["flags"] | (0 if tuned["flags"] & 8 else 4)
    reps = max(3, a.steps // 4)
    same, _ = timed(lambda: run(schedule="heuristic", **dict(tuned, flags=plain_flags)), reps, 1)
    plain_same = float(np.mean(same))
    # the reference's own root order: ids after its kcore recode (degeneracy
    # order, degree-sorted inside each shell), taken as given
    kc, _ = timed(lambda: run(schedule="given", **tuned), reps, 1)
    kcore_ms = float(np.mean(kc))
    extras = {"schedules": {
        "plain_kcore_order_ms": kcore_ms, "plain_heuristic_ms": plain_same, "learned_ms": step_ms,
        "learned_vs_plain": kcore_ms / step_ms, "learned_vs_degree_core_heuristic": plain_same / step_ms,
        "plain_default_launch_ms": float(np.mean(plain_ms)),
        "note": "plain = the reference's root order (its kcore tool's degeneracy order, degree-sorted inside each "
                "shell: the 'plain degree/core heuristic'); every ratio compares runs that differ in the order "
                "alone (same launch parameters and flags). degree_core_heuristic orders roots by descending "
                "degree x core number. plain_default_launch_ms: the heuristic order with the default launch",
        "tuned": tuned, "tuning_log": [[c, round(t, 3)] for c, t in tlog]}}
    e2e, cpu = None, None
    if not a.no_extras:
        e2e = e2e_leg(a, g, roots, tuned, total, dev, local, world, torch, models, dist)
    if not a.no_extras and world == 1:
        hs, _ = timed(lambda: run(schedule="heuristic", split=True, **dict(tuned, flags=1, granularity=4)), 3, 1)
        extras["schedules"]["heuristic_split_ms"] = float(np.mean(hs))
        gs, _ = timed(lambda: run(flags=1), 3, 1)
        extras["schedules"]["given_order_ms"] = float(np.mean(gs))
        # the plain heuristic order with the tuned launch parameters: the schedule's own effect
        launch = {k: v for k, v in tuned.items() if k in ("warps_per_block", "chunk", "ctas_per_sm")}
        ps, _ = timed(lambda: run(schedule="heuristic", flags=1, **launch), 3, 1)
        extras["schedules"]["plain_heuristic_tuned_launch_ms"] = float(np.mean(ps))
        # ---- triangles on the same graph (heuristic splits)
        ctx.set_plan(Plan.preset(0))
        tri_step = lambda: run(schedule="heuristic", **dict(tuned, flags=1))  # noqa: E731
        tri_step()
        tri = count()
        tms, _ = timed(tri_step, 3, 1)
        extras["triangle"] = {"count": tri, "ms_per_step": float(np.mean(tms)),
                              "per_s": tri / (float(np.mean(tms)) / 1000.0)}
        # ---- maximal cliques on a power-law graph (Chung-Lu n=2^18, gamma 2.3, avg degree 16)
        cl = g2aimd.Graph.chung_lu(1 << 18, 2.3, 16.0, seed=a.seed + rank).degeneracy_recoded()
        crp = torch.from_numpy(cl.row_ptrs.view(np.int64)).to(dev)
        cci = torch.from_numpy(cl.cols.view(np.int32)).to(dev)
        mctx = Context(local)
        mctx.load_device(crp.data_ptr(), cci.data_ptr(), cl.n, cl.m)
        mctx.load_core(cl.core)
        mctx.set_model(CostModel.load(os.path.join(models, "mce.npz")))
        mrun = lambda **kw: mctx.mce_device(out.data_ptr(), HIST, stream=sptr, **kw)  # noqa: E731
        mrun(schedule="heuristic", flags=2)
        mwork = work_of(mctx)
        cliques = count()
        cur["ctx"] = mctx
        # one warp per root (no hand-off), then walks handing branches to idle
        # warps; each order under the same settings (the learned run's tuned ones
        # for the hand-off rows)
        mgiven, _ = timed(lambda: mrun(schedule="given", flags=1 | FLAG_NO_SPILL), 3, 1)
        mplain, _ = timed(lambda: mrun(schedule="heuristic", flags=1 | FLAG_NO_SPILL), 3, 1)
        mlplain, _ = timed(lambda: mrun(schedule="learned", flags=1 | FLAG_NO_SPILL), 3, 1)
        mtuned, _, _ = tune(lambda **kw: mrun(schedule="learned", **kw), {"flags": 1, "chunk": 1}, MCE_SPACE)
        mgh, _ = timed(lambda: mrun(schedule="given", **mtuned), 3, 1)
        mhand, _ = timed(lambda: mrun(schedule="heuristic", **mtuned), 3, 1)
        mms, mpass = timed(lambda: mrun(schedule="learned", **mtuned), 3, 1)
        assert count() == cliques
        cur["ctx"] = ctx
        mk = float(np.mean(mpass)) if mpass else None
        mstream = cl.mce_stream_bytes()
        ml = float(np.mean(mms))
        extras["mce_chung_lu"] = {
            "graph": {"n": cl.n, "m": cl.m, "gamma": 2.3, "avg_degree": 16},
            "stream_bytes": mstream, "stream_gbs": mstream / (mk / 1000.0) / 1e9 if mk else None,
            "maximal_cliques": cliques,
            "no_handoff_ms": {"kcore_order": float(np.mean(mgiven)), "heuristic": float(np.mean(mplain)),
                              "learned": float(np.mean(mlplain))},
            "handoff_ms": {"kcore_order": float(np.mean(mgh)), "heuristic": float(np.mean(mhand)), "learned": ml},
            "learned_ms": ml, "learned_vs_plain": float(np.mean(mgh)) / ml,
            "learned_vs_degree_core_heuristic": float(np.mean(mhand)) / ml,
            "learned_vs_plain_no_handoff": float(np.mean(mgiven)) / float(np.mean(mlplain)),
            "note": "plain = the reference's kcore root order; each ratio compares the same settings",
            "tuned": mtuned, "per_s": cliques / (ml / 1000.0), "kernel_ms": mk,
            "merge_model_bytes": mwork, "merge_model_gbs": mwork / (mk / 1000.0) / 1e9 if mk else None}
        if rank == 0 and world == 1:
            cs = cpu_sample(cl, a.cpu_sample_s / 2, os.cpu_count() or 1, what="mce")
            extras["mce_chung_lu"]["cpu_port_per_s"] = cs["value"]
        mctx.close()
        # ---- degeneracy order of the benchmark graph: host peeling vs device peeling
        t0 = time.perf_counter()
        perm_h, core_h = g.degeneracy_order()
        host_s = time.perf_counter() - t0
        with Context(local) as oc:
            oc.load(g)
            oc.degeneracy_order()  # warm-up (module load)
            t0 = time.perf_counter()
            perm_d, core_d = oc.degeneracy_order()
            dev_s = time.perf_counter() - t0
        extras["degeneracy_order"] = {"host_s": host_s, "device_s": dev_s, "speedup": host_s / dev_s,
                                      "equal": bool(np.array_equal(perm_h, perm_d) and np.array_equal(core_h, core_d))}
        # ---- the whole preparation (order + recode) of the raw graph: host vs device
        raw = g2aimd.Graph.rmat(a.scale, a.edge_factor, 0.57, 0.19, 0.19, seed=a.seed)
        t0 = time.perf_counter()
        host_rec = raw.degeneracy_recoded()
        host_rs = time.perf_counter() - t0
        with Context(local) as oc:
            oc.load(raw)
            oc.degeneracy_recode()  # warm-up (module load)
            oc.load(raw)
            t0 = time.perf_counter()
            oc.degeneracy_recode()
            dev_rs = time.perf_counter() - t0
            dev_rec = oc.copy_csr(raw.m)
        extras["degeneracy_order"].update({
            "recode_host_s": host_rs, "recode_device_s": dev_rs, "recode_speedup": host_rs / dev_rs,
            "recode_equal": bool(np.array_equal(dev_rec.row_ptrs, host_rec.row_ptrs)
                                 and np.array_equal(dev_rec.cols, host_rec.cols))})
        # ---- a batch of 64 power-law graphs, one launch per job
        extras["batch_chung_lu_64"] = c4_leg(Context, CostModel, Plan, models, local, a.seed + rank, torch, stream)
        # ---- C3 (maximal cliques of R-MAT with planted cliques) and C5 (R-MAT s26 ef28)
        for key, leg in (("c3_rmat_planted", lambda: c3_leg(a, local, torch, stream, reps=2, budget_ms=10000)),
                         ("c5_rmat_s26_ef28", lambda: c5_leg(a, local, torch, stream, k5_stride=65536,
                                                              mce_budget_ms=10000))):
            try:
                extras[key] = leg()
            except Exception as exc:  # a failed leg is reported, the headline line still prints
                extras[key] = {"error": f"{type(exc).__name__}: {exc}"}
        # ---- the same graph out of core: view bins against in-core runs
        if world == 1:
            extras["view_bins"] = view_legs(a, g, 2, 1)
        if rank == 0 and world == 1:
            cs = cpu_stride_sample(g, 16, os.cpu_count() or 1)
            cpu = {"value": cs["value"], "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                   "sample": f"the {cs['roots']} roots v % 16 == 0 of the same graph (every 16th root in "
                             f"degeneracy order, heaviest first), {cs['seconds']:.1f} s, plan-driven enumeration "
                             "with the reference planner's plan (oracle/g2_oracle.c, all host threads)"}
    peak, peak_kind = measured_peak()
    stream_bytes = g.clique_stream_bytes(4)
    achieved = stream_bytes / (kern_ms / 1000.0) / 1e9 if kern_ms else None
    prof = headline_profile() if (a.scale, a.edge_factor, a.seed) == (20, 16, 1) else {}
    csum = clk.summary()
    issue = None
    if prof.get("inst") and kern_ms and csum.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        slots = sms * 4 * csum["sm_mhz"] * 1e6 * (kern_ms / 1000.0)  # warp-instruction issue slots
        issue = {"warp_instructions": prof["inst"], "issue_slots": slots, "frac": prof["inst"] / slots,
                 "source": prof["file"] + " (instructions per launch, ncu); kernel time and SM clock live"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": step_ms_all, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": bench_config(a, g.n, g.m, world),
            "count": int(total), "schedule": "learned (cost-model order, autotuned launch parameters)",
            "features_note": "root features are computed once per loaded graph and cached; the timed step "
                             "includes the MLP scoring, splits and the device sort of the task list",
            "l2_flush": "512 MiB written before every timed step", "graph_gen_s": round(gen_s, 2),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": prof.get("traffic"),
                         "kernel": "match_kernel<1,0,6> (clique bitmap path), main pass", "kernel_ms": kern_ms,
                         "algorithmic_bytes": stream_bytes, "peak_kind": peak_kind,
                         "binding": "instruction issue (see issue.frac); the HBM fraction is far from binding",
                         "issue": issue,
                         "merge_model_bytes": work_bytes,
                         "merge_model_gbs": work_bytes / (kern_ms / 1000.0) / 1e9 if kern_ms else None},
            "clocks": csum, "gpu_launches": int(launches_per_step * a.steps),
            "e2e": e2e, "cpu_baseline": cpu, "extras": extras,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        torch.distributed.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.leg == "c5":
        run_c5_leg(a)
    elif a.leg == "c3":
        run_c3_leg(a)
    elif a.leg == "walk":
        run_walk_leg(a)
    elif a.leg == "c4":
        run_c4_leg(a)
    elif a.leg == "mce":
        run_mce_leg(a)
    elif a.leg == "view":
        run_view_leg(a)
    elif a.leg == "view-host":
        run_view_host_leg(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
