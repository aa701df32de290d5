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
        L.orc_gen_rmat.argtypes = [u32, u32, C.c_double, C.c_double, C.c_double, u64, C.POINTER(vp),
                                   C.POINTER(vp), C.POINTER(u64)]
        L.orc_gen_rmat.restype = i32
        L.orc_free.argtypes = [vp]
        L.orc_free.restype = None
        L.orc_degeneracy_recode.argtypes = [vp, vp, u64, vp, vp, vp]
        L.orc_degeneracy_recode.restype = i32
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


class CSR:
    """A CSR graph held by the oracle alone (row_ptrs uint64, cols uint32), so
    that a CPU measurement can build its input without the library."""

    def __init__(self, row_ptrs, cols, core=None):
        self.row_ptrs, self.cols, self.core = row_ptrs, cols, core

    @property
    def n(self):
        return self.row_ptrs.size - 1

    @property
    def m(self):
        return self.cols.size


def gen_rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=1):
    """The seeded R-MAT graph of the library's generator (same ids, same rows)."""
    rp, ci, m = C.c_void_p(), C.c_void_p(), C.c_uint64()
    rc = lib().orc_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(rp), C.byref(ci), C.byref(m))
    if rc != 0:
        raise RuntimeError(f"orc_gen_rmat failed: {rc}")
    n = 1 << scale
    row_ptrs = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_uint64)), shape=(n + 1,)).copy()
    cols = np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_uint32)), shape=(max(m.value, 1),))[:m.value].copy()
    lib().orc_free(rp)
    lib().orc_free(ci)
    return CSR(row_ptrs, cols)


def degeneracy_recoded(g):
    """g with ids in the reference kcore tool's order (core numbers attached)."""
    orp = np.zeros(g.n + 1, np.uint64)
    oci = np.zeros(max(g.m, 1), np.uint32)
    core = np.zeros(g.n, np.uint32)
    rc = lib().orc_degeneracy_recode(_p(g.row_ptrs), _p(g.cols), g.n, _p(orp), _p(oci), _p(core))
    if rc != 0:
        raise RuntimeError(f"orc_degeneracy_recode failed: {rc}")
    return CSR(orp, oci[:g.m], core)


class PresetPlan:
    """A preset query's plan from the planner restatement (plan_oracle.py), in
    the form orc.match takes (k and flat())."""

    def __init__(self, query_id):
        import plan_oracle
        self.p = plan_oracle.preset_plan(query_id)
        self.k = self.p["k"]

    def flat(self):
        k, p = self.k, self.p
        bn = np.zeros(k * k, np.uint32)
        cond = np.zeros(k * k * 2, np.uint32)
        for i in range(k):
            for j, b in enumerate(p["bn"][i]):
                bn[i * k + j] = b
            for j, (op, w) in enumerate(p["cond"][i]):
                cond[(i * k + j) * 2] = op
                cond[(i * k + j) * 2 + 1] = w
        return (np.array(p["order"], np.uint32), np.array(p["id2order"], np.uint32),
                np.array([len(b) for b in p["bn"]], np.uint32), bn,
                np.array([len(c) for c in p["cond"]], np.uint32), cond)
