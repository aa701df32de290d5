"""Build libg2aimd.so (CUDA kernels for sm_100a + host C++) in-tree.

    python g2-aimd_b200/build.py          # incremental
    python g2-aimd_b200/build.py --clean

The library lands next to this file (g2-aimd_b200/libg2aimd.so) and is loaded
by g2aimd._lib through ctypes.  Every .cu file is compiled with
`-gencode arch=compute_100a,code=sm_100a -lineinfo`; there is no other target.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libg2aimd.so")
WORKER = os.path.join(HERE, "g2_worker")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH + INC
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-pthread", "-march=x86-64-v2"] + INC


MAIN = os.path.join(CSRC, "host", "worker_main.cpp")


def sources():
    cu, cpp = [], []
    for d, _, fs in os.walk(CSRC):
        for f in sorted(fs):
            p = os.path.join(d, f)
            if f.endswith(".cu"):
                cu.append(p)
            elif f.endswith(".cpp") and p != MAIN:
                cpp.append(p)
    return cu, cpp


def headers():
    hs = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    for d, _, fs in os.walk(CSRC):
        hs += [os.path.join(d, f) for f in fs if f.endswith((".cuh", ".h"))]
    return hs


def newer(src, dst, deps):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return os.path.getmtime(src) > t or any(os.path.getmtime(h) > t for h in deps)


def run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(verbose=False, ptxas_v=False):
    os.makedirs(OBJ, exist_ok=True)
    cu, cpp = sources()
    hs = headers()
    objs = []
    for s in cu:
        o = os.path.join(OBJ, os.path.relpath(s, CSRC).replace(os.sep, "_") + ".o")
        if newer(s, o, hs):
            extra = ["-Xptxas", "-v"] if ptxas_v else []
            run([NVCC] + NVFLAGS + extra + ["-c", s, "-o", o], verbose)
        objs.append(o)
    for s in cpp:
        o = os.path.join(OBJ, os.path.relpath(s, CSRC).replace(os.sep, "_") + ".o")
        if newer(s, o, hs):
            run([CXX] + CXXFLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"], verbose)
    # the reference-style command-line driver (drop-in for `bk` / `run`)
    if newer(MAIN, WORKER, hs) or os.path.getmtime(LIB) > os.path.getmtime(WORKER):
        run([CXX] + CXXFLAGS + [MAIN, "-o", WORKER, "-L", HERE, "-lg2aimd", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/smem use per kernel")
    a = ap.parse_args()
    if a.clean:
        shutil.rmtree(OBJ, ignore_errors=True)
        if os.path.exists(LIB):
            os.remove(LIB)
    print(build(a.verbose, a.ptxas_v))


if __name__ == "__main__":
    sys.exit(main())
