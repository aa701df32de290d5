"""Sanitizer builds of the host code: race detection for the threaded view code
(ThreadSanitizer), memory and undefined-behaviour checks (ASan + UBSan) for it
and for the graph and planner code.  Race detection: tests/tsan_views.cpp is
built with ThreadSanitizer together with csrc/host/view_host.cpp and run over
every threaded path (row passes, radius-1 walk, ego filter, bin planning on
several threads); any report fails the test."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_threaded_view_code_is_race_free(tmp_path):
    exe = tmp_path / "tsan_views"
    build = subprocess.run(
        ["g++", "-O1", "-g", "-std=c++17", "-fsanitize=thread", "-pthread", "-I", os.path.join(ROOT, "include"),
         "-I", os.path.join(ROOT, "g2-aimd_b200", "csrc"), os.path.join(HERE, "tsan_views.cpp"),
         os.path.join(ROOT, "g2-aimd_b200", "csrc", "host", "view_host.cpp"), "-o", str(exe)],
        capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, TSAN_OPTIONS="halt_on_error=1 exitcode=66"))
    assert run.returncode == 0, run.stderr[-4000:]
    assert "ThreadSanitizer" not in run.stderr
    assert run.stdout.count("mode") == 4


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_view_code_is_memory_safe(tmp_path):
    """The same paths under AddressSanitizer and UndefinedBehaviorSanitizer: no
    out-of-bounds access, leak or undefined behaviour in building views and bins
    (the views go to the GPU as they are)."""
    exe = tmp_path / "asan_views"
    build = subprocess.run(
        ["g++", "-O1", "-g", "-std=c++17", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
         "-pthread", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "g2-aimd_b200", "csrc"),
         os.path.join(HERE, "tsan_views.cpp"), os.path.join(ROOT, "g2-aimd_b200", "csrc", "host", "view_host.cpp"),
         "-o", str(exe)],
        capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1"))
    assert run.returncode == 0, run.stderr[-4000:]
    assert run.stdout.count("mode") == 4


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_graph_and_plan_host_code_is_memory_safe(tmp_path):
    """Generators, .bin / .vbmap / SNAP I/O, degeneracy order and recode and the
    planner under AddressSanitizer + UBSan (tests/sanitize_host.cpp)."""
    exe = tmp_path / "asan_host"
    host = os.path.join(ROOT, "g2-aimd_b200", "csrc", "host")
    build = subprocess.run(
        ["g++", "-O1", "-g", "-std=c++17", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
         "-pthread", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "g2-aimd_b200", "csrc"),
         os.path.join(HERE, "sanitize_host.cpp"), os.path.join(host, "graph_host.cpp"),
         os.path.join(host, "plan_host.cpp"), "-o", str(exe)],
        capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1"))
    assert run.returncode == 0, run.stderr[-4000:]
    assert "host ok" in run.stdout and "24 presets" in run.stdout, run.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_graph_host_threads_are_race_free(tmp_path):
    """The generators and the SNAP reader fan out over host threads: the same
    driver under ThreadSanitizer."""
    exe = tmp_path / "tsan_host"
    host = os.path.join(ROOT, "g2-aimd_b200", "csrc", "host")
    build = subprocess.run(
        ["g++", "-O1", "-g", "-std=c++17", "-fsanitize=thread", "-pthread", "-I", os.path.join(ROOT, "include"),
         "-I", os.path.join(ROOT, "g2-aimd_b200", "csrc"), os.path.join(HERE, "sanitize_host.cpp"),
         os.path.join(host, "graph_host.cpp"), os.path.join(host, "plan_host.cpp"), "-o", str(exe)],
        capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, TSAN_OPTIONS="halt_on_error=1 exitcode=66", G2_HOST_THREADS="6"))
    assert run.returncode == 0, run.stderr[-4000:]
    assert "ThreadSanitizer" not in run.stderr and "host ok" in run.stdout


@pytest.mark.skipif(shutil.which("g++") is None or shutil.which("gcc") is None, reason="needs gcc and g++")
def test_oracle_is_memory_safe(tmp_path):
    """The CPU oracle, the checker every parity test relies on, under
    AddressSanitizer + UBSan on all of its entry points (tests/sanitize_oracle.cpp;
    OpenMP threads included, so no ThreadSanitizer run here)."""
    san = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fopenmp", "-g", "-O1"]
    obj = tmp_path / "oracle.o"
    cc = subprocess.run(["gcc", *san, "-std=c11", "-c", os.path.join(ROOT, "oracle", "g2_oracle.c"), "-o", str(obj)],
                        capture_output=True, text=True, timeout=600)
    assert cc.returncode == 0, cc.stderr
    exe = tmp_path / "asan_oracle"
    host = os.path.join(ROOT, "g2-aimd_b200", "csrc", "host")
    build = subprocess.run(
        ["g++", *san, "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "include"),
         os.path.join(HERE, "sanitize_oracle.cpp"), str(obj), os.path.join(host, "graph_host.cpp"),
         os.path.join(host, "plan_host.cpp"), "-o", str(exe)],
        capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1"))
    assert run.returncode == 0, run.stderr[-4000:]
    assert "oracle ok" in run.stdout, run.stdout
