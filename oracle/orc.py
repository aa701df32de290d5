"""ctypes wrapper of oracle/liborc.so (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this module.  It is the checker, never the thing measured or shipped.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "liborc.so"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, u64, i32, u32 = C.c_void_p, C.c_uint64, C.c_int, C.c_uint32
        L.orc_mce.argtypes = [vp, vp, u64, vp, u64, i32, C.POINTER(u64), vp, u32, C.POINTER(u64), vp, vp]
        L.orc_mce.restype = i32
        L.orc_match.argtypes = [vp, vp, u64, vp, u64, i32, u32, vp, vp, vp, vp, vp, vp, C.POINTER(u64),
                                C.POINTER(u64), vp]
        L.orc_match.restype = i32
        L.orc_embeddings.argtypes = [vp, vp, u64, u32, vp, C.POINTER(u64)]
        L.orc_embeddings.restype = i32
        L.orc_mce_bruteforce.argtypes = [vp, vp, u64, C.POINTER(u64), vp, u32]
        L.orc_mce_bruteforce.restype = i32
        L.orc_kcore.argtypes = [vp, vp, u64, vp, vp]
        L.orc_kcore.restype = C.c_int64
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def mce(g, roots=None, threads=1, hist_len=256, per_root=False):
    """Reference-rule MCE: dict(count, hist, work[, root_nodes, root_work])."""
    r = None if roots is None else np.ascontiguousarray(roots, dtype=np.uint32)
    nr = g.n if r is None else r.size
    cnt, work = C.c_uint64(), C.c_uint64()
    hist = np.zeros(hist_len, np.uint64)
    rn = np.zeros(nr, np.uint64) if per_root else None
    rw = np.zeros(nr, np.uint64) if per_root else None
    rc = lib().orc_mce(_p(g.row_ptrs), _p(g.cols), g.n, _p(r), nr, threads, C.byref(cnt), _p(hist), hist_len,
                       C.byref(work), _p(rn), _p(rw))
    if rc not in (0,):
        raise RuntimeError(f"orc_mce failed: {rc}")
    out = {"count": cnt.value, "hist": hist, "work": work.value}
    if per_root:
        out["root_nodes"] = rn
        out["root_work"] = rw
    return out


def match(g, plan, roots=None, threads=1, per_root=False):
    """Plan-driven count (reference plain path): dict(count, work[, root_counts])."""
    order, id2order, bn_count, bn, cond_count, cond = plan.flat()
    r = None if roots is None else np.ascontiguousarray(roots, dtype=np.uint32)
    nr = g.n if r is None else r.size
    cnt, work = C.c_uint64(), C.c_uint64()
    rcn = np.zeros(nr, np.uint64) if per_root else None
    rc = lib().orc_match(_p(g.row_ptrs), _p(g.cols), g.n, _p(r), nr, threads, plan.k, _p(order), _p(id2order),
                         _p(bn_count), _p(bn), _p(cond_count), _p(cond), C.byref(cnt), C.byref(work), _p(rcn))
    if rc != 0:
        raise RuntimeError(f"orc_match failed: {rc}")
    out = {"count": cnt.value, "work": work.value}
    if per_root:
        out["root_counts"] = rcn
    return out


def embeddings(g, k, edges):
    """Injective edge-preserving maps of the query into g (brute force)."""
    adj = np.zeros((k, k), np.uint32)
    for a, b in edges:
        adj[a, b] = adj[b, a] = 1
    out = C.c_uint64()
    rc = lib().orc_embeddings(_p(g.row_ptrs), _p(g.cols), g.n, k, _p(np.ascontiguousarray(adj)), C.byref(out))
    if rc != 0:
        raise RuntimeError(f"orc_embeddings failed: {rc}")
    return out.value


def mce_bruteforce(g, hist_len=64):
    cnt = C.c_uint64()
    hist = np.zeros(hist_len, np.uint64)
    rc = lib().orc_mce_bruteforce(_p(g.row_ptrs), _p(g.cols), g.n, C.byref(cnt), _p(hist), hist_len)
    if rc != 0:
        raise RuntimeError(f"orc_mce_bruteforce failed: {rc}")
    return cnt.value, hist


def kcore(g):
    """(peel order, core numbers, kmax) as kmeans/kcore.cpp computes them."""
    order = np.zeros(g.n, np.uint32)
    core = np.zeros(g.n, np.uint32)
    kmax = lib().orc_kcore(_p(g.row_ptrs), _p(g.cols), g.n, _p(order), _p(core))
    return order, core, int(kmax)
