"""bench.py's host-only leg (view shapes, no GPU) runs and reports one JSON line
whose view sizes follow the shapes: full balls >= upper balls >= forward rows,
and ego rows below the rows they filter."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_view_host_leg_small():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--leg", "view-host", "--scale", "10",
                          "--edge-factor", "8"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    k = {key.split("/", 1)[1]: v for key, v in line.items() if key.startswith("k4_rmat_s10/")}
    assert set(k) == {"full", "upper", "forward", "forward+ego"}
    assert k["full"]["view_entries"] >= k["upper"]["view_entries"] >= k["forward"]["view_entries"]
    assert k["forward+ego"]["view_entries"] <= k["forward"]["view_entries"]
    mce = line["mce_chung_lu_2^18/full"], line["mce_chung_lu_2^18/full+ego"]
    assert mce[1]["view_entries"] < mce[0]["view_entries"] and mce[0]["bins"] == mce[1]["bins"]
