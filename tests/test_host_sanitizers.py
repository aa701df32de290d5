"""Sanitizer builds of the host code: race detection (ThreadSanitizer) and
memory / undefined-behaviour checks (AddressSanitizer + UBSan).  Drivers in
this directory call every host entry point on graphs large enough for the
threaded paths; any sanitizer report fails the test.
  tests/tsan_views.cpp      view builder, bin planner, view C entry points
  tests/sanitize_host.cpp   generators, .bin / .vbmap / SNAP I/O, order, recode, planner
  tests/sanitize_oracle.cpp the CPU oracle (the checker of every parity test)
  g2_worker's host-only modes, device entry points stubbed (tests/worker_gpu_stubs.cpp)"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
HOST = os.path.join(ROOT, "g2-aimd_b200", "csrc", "host")
TSAN = ["-fsanitize=thread"]
ASAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all"]

pytestmark = pytest.mark.skipif(shutil.which("g++") is None or shutil.which("gcc") is None,
                                reason="needs gcc and g++")


def build(exe, sources, san, extra=()):
    cmd = ["g++", "-O1", "-g", "-std=c++17", "-pthread", *san, *extra, "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "g2-aimd_b200", "csrc"), *sources, "-o", str(exe)]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr


def run(exe, args=(), **env):
    env = dict(os.environ, TSAN_OPTIONS="halt_on_error=1 exitcode=66", ASAN_OPTIONS="detect_leaks=1", **env)
    out = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-4000:]
    assert "Sanitizer" not in out.stderr, out.stderr[-4000:]
    return out.stdout


VIEWS = [os.path.join(HERE, "tsan_views.cpp"), os.path.join(HOST, "view_host.cpp")]
GRAPH = [os.path.join(HERE, "sanitize_host.cpp"), os.path.join(HOST, "graph_host.cpp"),
         os.path.join(HOST, "plan_host.cpp")]


def test_threaded_view_code_is_race_free(tmp_path):
    """Row passes, the atomic radius-1 walk, the ego filter and range-parallel
    bin plans on several threads."""
    build(tmp_path / "t", VIEWS, TSAN)
    assert run(tmp_path / "t").count("mode") == 4


def test_view_code_is_memory_safe(tmp_path):
    """The same paths and the view C entry points (the views go to the GPU as
    they are)."""
    build(tmp_path / "a", VIEWS, ASAN)
    assert "rebalanced bins" in run(tmp_path / "a")


def test_graph_and_plan_host_code_is_memory_safe(tmp_path):
    build(tmp_path / "a", GRAPH, ASAN)
    out = run(tmp_path / "a", [tmp_path])
    assert "host ok" in out and "24 presets" in out, out


def test_graph_host_threads_are_race_free(tmp_path):
    """The generators and the SNAP reader fan out over host threads."""
    build(tmp_path / "t", GRAPH, TSAN)
    assert "host ok" in run(tmp_path / "t", [tmp_path], G2_HOST_THREADS="6")


def test_oracle_is_memory_safe(tmp_path):
    """OpenMP threads included, so ASan + UBSan only (no ThreadSanitizer)."""
    obj = tmp_path / "oracle.o"
    cc = subprocess.run(["gcc", "-O1", "-g", "-std=c11", "-fopenmp", *ASAN, "-c",
                         os.path.join(ROOT, "oracle", "g2_oracle.c"), "-o", str(obj)],
                        capture_output=True, text=True, timeout=600)
    assert cc.returncode == 0, cc.stderr
    build(tmp_path / "o", [os.path.join(HERE, "sanitize_oracle.cpp"), str(obj), os.path.join(HOST, "graph_host.cpp"),
                           os.path.join(HOST, "plan_host.cpp")], ASAN, ["-fopenmp"])
    assert "oracle ok" in run(tmp_path / "o")


def test_worker_host_modes_are_memory_safe(tmp_path):
    """g2_worker's -prep, -recode and -plan under AddressSanitizer + UBSan (device
    entry points stubbed: these modes use none)."""
    build(tmp_path / "w", [os.path.join(HOST, "worker_main.cpp"), os.path.join(HERE, "worker_gpu_stubs.cpp"),
                           os.path.join(HOST, "graph_host.cpp"), os.path.join(HOST, "plan_host.cpp"),
                           os.path.join(HOST, "view_host.cpp")], ASAN)
    txt = tmp_path / "g.txt"
    with open(txt, "w") as f:
        f.write("# toy\n")
        for a in range(300):
            for b in (a * 7 % 300, a * 13 % 300, (a + 1) % 300):
                f.write(f"{a + 10} {b + 10}\n")
    run(tmp_path / "w", ["-dg", txt, "-prep", 1])
    run(tmp_path / "w", ["-dg", tmp_path / "g.bin", "-recode", 1, "-o", tmp_path / "r.bin", "-nb", 3])
    out = run(tmp_path / "w", ["-dg", tmp_path / "r.bin", "-q", 24, "-plan", 1, "-m", 0.000002, "-ds", 1, "-cn", 2,
                               "-dr", 1])
    assert "wrote" in out and int(out.split("view bins: ")[1].split()[0]) > 1
    run(tmp_path / "w", ["-dg", tmp_path / "r.bin", "-h", 2, "-plan", 1, "-m", 0.000004, "-t", 3])
