"""Train the root-cost models shipped in g2-aimd_b200/models/.

    python -m g2aimd.train_costmodel [--out DIR] [--quick]

For each workload the plain persistent kernel (roots in id order, no splits)
logs the SM cycles of every root on seeded synthetic graphs whose seeds differ
from every test and benchmark graph; the library's own tensor-core kernels
(g2_model_train) then fit the MLP to log1p(cycles) from the 8 root features.

  k4   4-clique plan (preset 24) on R-MAT graphs, edge factor 16, scales 16-19
  mce  maximal cliques on Chung-Lu power-law graphs (2^15-2^17 vertices) and
       R-MAT graphs of scale 11-13 (larger R-MAT graphs have too many maximal
       cliques to enumerate)
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from .context import Context, CostModel, Plan
from .graph import Graph

HERE = os.path.dirname(os.path.abspath(__file__))
MODELS = os.path.join(os.path.dirname(HERE), "models")


def training_graphs(task, quick=False):
    if task == "k4":
        scales = [14, 15] if quick else [16, 17, 18, 19]
        for i, s in enumerate(scales):
            yield Graph.rmat(s, 16, seed=1000 + i).degeneracy_recoded()
    else:
        sizes = [1 << 14, 1 << 15] if quick else [1 << 15, 1 << 16, 1 << 17]
        for i, n in enumerate(sizes):
            for gam in (2.3, 2.5):
                yield Graph.chung_lu(n, gam, 16.0, seed=2000 + 10 * i + int(gam * 10)).degeneracy_recoded()
        for s in ([10, 11] if quick else [11, 12, 13]):
            yield Graph.rmat(s, 16, seed=3000 + s).degeneracy_recoded()


def collect(ctx, task, quick=False):
    Xs, cs, info = [], [], []
    plan = Plan.preset(24)
    for g in training_graphs(task, quick):
        ctx.load(g)
        ctx.load_core(g.core)
        cost = np.zeros(g.n, np.uint64)
        t = time.perf_counter()
        if task == "k4":
            ctx.match(plan, root_cost=cost)
        else:
            ctx.mce(root_cost=cost)
        keep = g.degrees() > 0
        Xs.append(ctx.root_features()[keep])
        cs.append(cost[keep].astype(np.float32))
        info.append({"graph": g.name, "n": g.n, "m": g.m, "roots": int(keep.sum()),
                     "seconds": round(time.perf_counter() - t, 3)})
    return np.concatenate(Xs), np.concatenate(cs), info


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=MODELS)
    ap.add_argument("--quick", action="store_true", help="small graphs (tests)")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--tasks", default="k4,mce")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    with Context(0) as ctx:
        for task in a.tasks.split(","):
            X, c, info = collect(ctx, task, a.quick)
            t = time.perf_counter()
            m = CostModel.train(ctx, X, c, epochs=a.epochs, batch=2048, lr=3e-3, seed=17)
            meta = {"task": task, "rows": int(X.shape[0]), "epochs": a.epochs, "train_s": round(time.perf_counter() - t, 2),
                    "loss_first": float(m.losses[0]), "loss_last": float(m.losses[-1]), "graphs": info}
            path = os.path.join(a.out, f"{task}.npz")
            np.savez(path, params=m.params, norm=m.norm, meta=json.dumps(meta))
            print(json.dumps(meta))


if __name__ == "__main__":
    main()
