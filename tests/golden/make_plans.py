"""Regenerate tests/golden/plans.json from the REFERENCE query planner.

Run `make -C oracle ref` first (it builds oracle/_ref/ref_plan from the
reference's common/graph.h + system/plan.h with bliss rebuilt from source),
then `python tests/golden/make_plans.py`.  The JSON holds, for every preset
query id, the plan exactly as the reference computes it.
"""
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
QUERIES = list(range(0, 19)) + list(range(23, 28))

if __name__ == "__main__":
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_plan")
    out = json.loads(subprocess.check_output([exe] + [str(q) for q in QUERIES]))
    with open(os.path.join(HERE, "plans.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", len(out), "plans")
