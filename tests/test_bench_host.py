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


def test_reference_arm_runs_without_the_library():
    """`bench.py --impl reference` builds its graph and plan in the oracle and
    never loads libg2aimd.so; over its timed steps it covers every root once,
    so its count is the whole graph's (checked against the oracle here)."""
    code = (
        "import sys, runpy, json\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--scale', '11', '--steps', '4', '--warmup', '2']\n"
        f"runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'lib_loaded': 'libg2aimd.so' in maps, 'orc_loaded': 'liborc.so' in maps}))\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    lines = [json.loads(x) for x in out.stdout.strip().splitlines() if x.startswith("{")]
    ref, maps = lines[-2], lines[-1]
    assert ref["impl"] == "reference" and not maps["lib_loaded"] and maps["orc_loaded"]
    assert ref["roots_covered"] == 1 << 11
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    g = orc.degeneracy_recoded(orc.gen_rmat(11, 16, seed=1))
    assert ref["count"] == orc.match(g, orc.PresetPlan(24), threads=4)["count"]
    assert ref["config"]["graph"] == {"n": g.n, "m": g.m, "seed": 1}
