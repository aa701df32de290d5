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
Inputs (ids in degeneracy order): R-MAT scale 20 edge factor 16 (4-clique and
triangle), Chung-Lu 2^18 gamma 2.3 degree 16 and ER(2000, 0.01) + 5 K12
(maximal cliques).  Each run has a time limit; a reference run that does not
finish is reported as such.
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


def parse(out):
    t = sum(float(x) for x in re.findall(r"In-memory Execution Time, elapsed_time=([0-9.]+)ms", out))
    cl = [int(x) for x in re.findall(r"Total No\. of Cliques: (\d+)", out)]
    tc = re.findall(r"^Total counts: (\d+)", out, flags=re.M)
    tot = re.findall(r"total time, elapsed_time=([0-9.]+)ms", out)
    return {"in_memory_ms": t, "cliques": sum(cl) if cl else None, "counts": int(tc[-1]) if tc else None,
            "total_ms": float(tot[-1]) if tot else None}


def run(cmd, limit):
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=limit)
        r = parse(p.stdout)
        r["rc"] = p.returncode
        if "Host overflow" in p.stdout:
            r["note"] = "host overflow (reference cannot complete)"
        return r
    except subprocess.TimeoutExpired:
        return {"rc": None, "note": f"did not finish within {limit} s"}


def main():
    import g2aimd
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--limit", type=int, default=600)
    a = ap.parse_args()
    ref_run, ref_bk = os.path.join(HERE, "_ref", "ref_run"), os.path.join(HERE, "_ref", "ref_bk")
    ours = os.path.join(ROOT, "g2-aimd_b200", "g2_worker")
    work = tempfile.mkdtemp(prefix="g2ref_")
    graphs = {
        "rmat20": g2aimd.Graph.rmat(20, 16, seed=1).degeneracy_recoded(),
        "chunglu18": g2aimd.Graph.chung_lu(1 << 18, 2.3, 16.0, seed=1).degeneracy_recoded(),
        "er2000_k12": g2aimd.Graph.er(2000, 0.01, planted=5, planted_size=12, seed=7).degeneracy_recoded(),
    }
    jobs = [("rmat20", "q24"), ("rmat20", "q0"), ("chunglu18", "mce"), ("er2000_k12", "mce")]
    results = []
    for name, job in jobs:
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
        res = {"graph": name, "n": g.n, "m": g.m, "job": job, "reference_gpu": r, "g2_worker": o}
        print(json.dumps(res), flush=True)
        results.append(res)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(results, f, indent=1)


if __name__ == "__main__":
    main()
