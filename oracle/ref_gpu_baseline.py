"""Run the reference's own GPU build and g2_worker on the same inputs (baseline).

    make -C oracle ref-gpu          # builds oracle/_ref/ref_run and ref_bk here
    python oracle/ref_gpu_baseline.py [--out results.json]

Writes each input graph as `.bin` + one-bin `.bin.2.hop.vbmap` (the reference's
formats), then runs, with the same flags,
  reference:  oracle/_ref/ref_run -dg G.bin -q Q -m 1     (app_gmatch, as shipped)
              oracle/_ref/ref_bk  -dg G.bin -h 2 -m 1     (app_BK, as shipped)
  this repo:  g2-aimd_b200/g2_worker  (same flags, same result lines)
and parses "Total counts:" / "Total No. of Cliques:" and the
"In-memory Execution Time" lines (device loop only, both programs).
Inputs (ids in degeneracy order, the generators in g2aimd.graph):
  er2000_k12   ER(2000, 0.01) + 5 K12, seed 7               maximal cliques
  rmat20       R-MAT scale 20 edge factor 16, seed 1          triangles, 4-, 5-cliques
  rmat16       R-MAT scale 16 edge factor 16, seed 3          4-cycles, diamonds, 4-, 5-cliques
  chunglu18    Chung-Lu 2^18 gamma 2.3 degree 16, seed 1      maximal cliques, triangles
  cl_*         three Chung-Lu graphs shaped like the 64-graph batch members
               (n 5e3 / 5e4 / 2e5)                            maximal cliques, triangles,
                                                              4-cycles, diamonds
  rmat13_k     R-MAT scale 13 edge factor 16 + 20 planted cliques of 20-60
               vertices, seed 5                              maximal cliques
Each run has a time limit; a reference run that does not finish is reported as
such.  A reference GMatch run that printed a '--- chunk' line retried a chunk
after a buffer overflow and double counts (its iterationFailed is a no-op), so
such a count is marked untrusted; so is any run that printed 'Host overflow'.
A clique count is also marked untrusted when the reference's deepest stored
level cannot fit its 32-bit record indices (Index = unsigned int,
common/gpu_env.h:79, used for the buffer tails in system/buffer.h): for a
k-clique plan that level holds every (k-1)-clique with k-1 vertices each, so
the (k-1)-clique count of the same graph (an earlier job) times k-1 must stay
below 2^32; beyond it the tails wrap and records overwrite each other without
any message.
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "g2-aimd_b200"))


# graph name -> generator call (ids are then put in degeneracy order)
GRAPHS = [
    ("er2000_k12", "Graph.er(2000, 0.01, planted=5, planted_size=12, seed=7)",
     lambda G: G.er(2000, 0.01, planted=5, planted_size=12, seed=7)),
    ("rmat20", "Graph.rmat(20, 16, seed=1)", lambda G: G.rmat(20, 16, seed=1)),
    ("rmat16", "Graph.rmat(16, 16, seed=3)", lambda G: G.rmat(16, 16, seed=3)),
    ("chunglu18", "Graph.chung_lu(1 << 18, 2.3, 16.0, seed=1)", lambda G: G.chung_lu(1 << 18, 2.3, 16.0, seed=1)),
    ("cl_5k", "Graph.chung_lu(5000, 2.5, 20.0, seed=11)", lambda G: G.chung_lu(5000, 2.5, 20.0, seed=11)),
    ("cl_50k", "Graph.chung_lu(50000, 2.2, 30.0, seed=12)", lambda G: G.chung_lu(50000, 2.2, 30.0, seed=12)),
    ("cl_200k", "Graph.chung_lu(200000, 2.8, 10.0, seed=13)", lambda G: G.chung_lu(200000, 2.8, 10.0, seed=13)),
    ("rmat13_k", "Graph.rmat(13, 16, planted=20, pmin=20, pmax=60, seed=5)",
     lambda G: G.rmat(13, 16, planted=20, pmin=20, pmax=60, seed=5)),
]
JOBS = [("er2000_k12", "mce"), ("rmat20", "q24"), ("rmat20", "q0"), ("rmat20", "q25"),
        ("rmat16", "q1"), ("rmat16", "q2"), ("rmat16", "q24"), ("rmat16", "q25"),
        ("chunglu18", "mce"), ("chunglu18", "q0")] + \
       [(g, j) for g in ("cl_5k", "cl_50k", "cl_200k") for j in ("mce", "q0", "q1", "q2")] + \
       [("rmat13_k", "mce")]


# k-clique preset -> the (k-1)-clique preset whose matches the reference stores
# at its deepest level, and k - 1
CLIQUE_PREFIX = {"q24": ("q0", 3), "q25": ("q24", 4)}


def index_overflow(results, name, job):
    """Reason the reference's 32-bit record indices overflow on this job, or None."""
    if job not in CLIQUE_PREFIX:
        return None
    pre, width = CLIQUE_PREFIX[job]
    for r in results:
        if r["graph"] == name and r["job"] == pre and r["g2_worker"].get("counts") is not None:
            entries = r["g2_worker"]["counts"] * width
            if entries >= 1 << 32:
                return (f"level-{width} frontier of {entries} entries ({pre} matches x {width}) exceeds the "
                        "32-bit record indices")
    return None


def parse(out):
    t = sum(float(x) for x in re.findall(r"In-memory Execution Time, elapsed_time=([0-9.]+)ms", out))
    cl = [int(x) for x in re.findall(r"Total No\. of Cliques: (\d+)", out)]
    tc = re.findall(r"^Total counts: (\d+)", out, flags=re.M)
    tot = re.findall(r"total time, elapsed_time=([0-9.]+)ms", out)
    return {"in_memory_ms": t, "cliques": sum(cl) if cl else None, "counts": int(tc[-1]) if tc else None,
            "total_ms": float(tot[-1]) if tot else None, "chunk_retries": len(re.findall(r"--- chunk", out))}


def run(cmd, limit):
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=limit)
        r = parse(p.stdout)
        r["rc"] = p.returncode
        if "Host overflow" in p.stdout:
            r["note"] = "host overflow (reference cannot complete)"
        r["trusted"] = p.returncode == 0 and "Host overflow" not in p.stdout and r["chunk_retries"] == 0
        return r
    except subprocess.TimeoutExpired:
        return {"rc": None, "note": f"did not finish within {limit} s"}


def main():
    import g2aimd
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--limit", type=int, default=600)
    ap.add_argument("--only", default="", help="comma-separated graph names")
    a = ap.parse_args()
    ref_run, ref_bk = os.path.join(HERE, "_ref", "ref_run"), os.path.join(HERE, "_ref", "ref_bk")
    ours = os.path.join(ROOT, "g2-aimd_b200", "g2_worker")
    work = tempfile.mkdtemp(prefix="g2ref_")
    makers = {name: (text, fn) for name, text, fn in GRAPHS}
    jobs = JOBS if not a.only else [j for j in JOBS if j[0] in a.only.split(",")]
    graphs = {}
    results = []
    for name, job in jobs:
        if name not in graphs:
            graphs[name] = makers[name][1](g2aimd.Graph).degeneracy_recoded()
        g = graphs[name]
        path = os.path.join(work, f"{name}.bin")
        if not os.path.exists(path):
            g.write_bin(path)
            g.write_vbmap(path + ".2.hop.vbmap", 1)
        if job == "mce":
            args = ["-dg", path, "-h", "2", "-m", "1"]
            r = run([ref_bk] + args, a.limit)
            o = run([ours] + args, a.limit)
        else:
            args = ["-dg", path, "-q", job[1:], "-m", "1"]
            r = run([ref_run] + args, a.limit)
            o = run([ours] + args, a.limit)
        why = index_overflow(results, name, job)
        if why:
            r["trusted"] = False
            r["note"] = why
        res = {"graph": name, "make": makers[name][0], "n": g.n, "m": g.m, "job": job, "reference_gpu": r,
               "g2_worker": o}
        print(json.dumps(res), flush=True)
        results.append(res)
        if a.out:  # rewritten after every job, so a cut-off run keeps what finished
            with open(a.out, "w") as f:
                json.dump(results, f, indent=1)


if __name__ == "__main__":
    main()
