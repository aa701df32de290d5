"""CSR graphs in the reference's .bin layout (common/graph.h:360-398).

A Graph holds `row_ptrs` (uint64, n+1) and `cols` (uint32, m) as numpy arrays:
symmetric, sorted, deduplicated, no self loops.  Generation, I/O, degeneracy
ordering and recoding call libg2aimd.so's host functions.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _take(rp_p, ci_p, n, m):
    L = lib()
    rp = np.ctypeslib.as_array(C.cast(rp_p, C.POINTER(C.c_uint64)), shape=(n + 1,)).copy()
    ci = np.ctypeslib.as_array(C.cast(ci_p, C.POINTER(C.c_uint32)), shape=(max(m, 1),))[:m].copy()
    L.g2_free(rp_p)
    L.g2_free(ci_p)
    return rp, ci


class Graph:
    def __init__(self, row_ptrs, cols, name=""):
        self.row_ptrs = np.ascontiguousarray(row_ptrs, dtype=np.uint64)
        self.cols = np.ascontiguousarray(cols, dtype=np.uint32)
        self.name = name
        if self.row_ptrs.ndim != 1 or self.row_ptrs.size < 1 or int(self.row_ptrs[-1]) != self.cols.size:
            raise ValueError("row_ptrs[-1] must equal len(cols)")

    # ------------------------------------------------------------- basics
    @property
    def n(self) -> int:
        return self.row_ptrs.size - 1

    @property
    def m(self) -> int:
        return self.cols.size

    def degrees(self):
        return np.diff(self.row_ptrs).astype(np.int64)

    def neighbors(self, v):
        return self.cols[self.row_ptrs[v]:self.row_ptrs[v + 1]]

    def __repr__(self):
        return f"Graph({self.name or 'anon'}: n={self.n}, m={self.m})"

    # ----------------------------------------------------------- builders
    @staticmethod
    def from_edges(n, edges, name=""):
        """Symmetric, deduplicated CSR from an iterable of (u, v) pairs."""
        e = np.asarray(list(edges), dtype=np.int64).reshape(-1, 2)
        e = e[e[:, 0] != e[:, 1]]
        both = np.concatenate([e, e[:, ::-1]]) if e.size else e
        keys = np.unique(both[:, 0] * (1 << 32) + both[:, 1]) if both.size else np.zeros(0, np.int64)
        src, dst = keys >> 32, keys & 0xFFFFFFFF
        rp = np.zeros(n + 1, np.uint64)
        np.add.at(rp, src + 1, 1)
        return Graph(np.cumsum(rp).astype(np.uint64), dst.astype(np.uint32), name)

    @staticmethod
    def er(n, p, planted=0, planted_size=0, seed=1):
        rp, ci, nn, mm = C.c_void_p(), C.c_void_p(), C.c_uint64(), C.c_uint64()
        check(lib().g2_gen_er(n, p, planted, planted_size, seed, C.byref(rp), C.byref(ci), C.byref(nn),
                              C.byref(mm)), "g2_gen_er")
        return Graph(*_take(rp, ci, nn.value, mm.value), name=f"er{n}_{p}+{planted}xK{planted_size}_s{seed}")

    @staticmethod
    def rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, planted=0, pmin=0, pmax=0, seed=1):
        rp, ci, nn, mm = C.c_void_p(), C.c_void_p(), C.c_uint64(), C.c_uint64()
        check(lib().g2_gen_rmat(scale, edge_factor, a, b, c, planted, pmin, pmax, seed, C.byref(rp), C.byref(ci),
                                C.byref(nn), C.byref(mm)), "g2_gen_rmat")
        return Graph(*_take(rp, ci, nn.value, mm.value), name=f"rmat{scale}e{edge_factor}+{planted}_s{seed}")

    @staticmethod
    def chung_lu(n, gamma, avg_degree, seed=1):
        rp, ci, nn, mm = C.c_void_p(), C.c_void_p(), C.c_uint64(), C.c_uint64()
        check(lib().g2_gen_chunglu(n, gamma, avg_degree, seed, C.byref(rp), C.byref(ci), C.byref(nn),
                                   C.byref(mm)), "g2_gen_chunglu")
        return Graph(*_take(rp, ci, nn.value, mm.value), name=f"cl{n}_g{gamma:.2f}_d{avg_degree:.1f}_s{seed}")

    # ---------------------------------------------------------------- I/O
    @staticmethod
    def read_bin(path):
        rp, ci, nn, mm = C.c_void_p(), C.c_void_p(), C.c_uint64(), C.c_uint64()
        check(lib().g2_read_bin(str(path).encode(), C.byref(rp), C.byref(ci), C.byref(nn), C.byref(mm)),
              f"read {path}")
        return Graph(*_take(rp, ci, nn.value, mm.value), name=str(path))

    @staticmethod
    def read_snap(path, preprocess=True):
        """SNAP text edge list (g2_read_snap); preprocess as the reference's
        Graph::Preprocess (dedupe, no self loops, isolated vertices dropped)."""
        rp, ci, nn, mm = C.c_void_p(), C.c_void_p(), C.c_uint64(), C.c_uint64()
        check(lib().g2_read_snap(str(path).encode(), int(bool(preprocess)), C.byref(rp), C.byref(ci),
                                 C.byref(nn), C.byref(mm)), f"read {path}")
        return Graph(*_take(rp, ci, nn.value, mm.value), name=str(path))

    def write_bin(self, path):
        check(lib().g2_write_bin(str(path).encode(), _ptr(self.row_ptrs), _ptr(self.cols), self.n, self.m),
              f"write {path}")

    def write_vbmap(self, path, nbins=1, bins=None):
        b = None if bins is None else np.ascontiguousarray(bins, dtype=np.uint32)
        check(lib().g2_write_vbmap(str(path).encode(), nbins, _ptr(b), self.n), f"write {path}")

    def read_vbmap(self, path):
        nb = C.c_uint32()
        bins = np.zeros(self.n, np.uint32)
        check(lib().g2_read_vbmap(str(path).encode(), self.n, C.byref(nb), _ptr(bins)), f"read {path}")
        return nb.value, bins

    # ----------------------------------------------------- views (out of core)
    def view(self, sources, radius=1, row_radius=None, min_root_degree=0, upper=False, forward=False, ego=False):
        """(view graph, local sources, global ids) of the ball of `radius` around
        `sources` (g2_view_materialize): ids ascending in global order, rows kept
        for vertices within row_radius (default: radius), restricted to the ball;
        upper: each source's ball walked through vertices above it; forward: rows
        keep only their entries above their own vertex; ego (radius 1): rows keep
        only edges inside some source's closed neighbourhood."""
        from ._lib import G2View
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        v = G2View()
        rr = radius if row_radius is None else row_radius
        check(lib().g2_view_materialize(_ptr(self.row_ptrs), _ptr(self.cols), self.n, _ptr(src), src.size,
                                        radius, rr, min_root_degree,
                                        int(bool(upper)) | 4 * int(bool(forward)) | 8 * int(bool(ego)),
                                        C.byref(v)),
              "g2_view_materialize")
        try:
            n, m, ns = v.n, v.m, v.nsrc
            rp = np.ctypeslib.as_array(v.row_ptrs, shape=(n + 1,)).copy()
            ci = np.ctypeslib.as_array(v.cols, shape=(max(m, 1),))[:m].copy()
            fo = np.ctypeslib.as_array(v.fwd_offsets, shape=(max(n, 1),))[:n].copy()
            lsrc = np.ctypeslib.as_array(v.sources, shape=(max(ns, 1),))[:ns].copy()
            ids = np.ctypeslib.as_array(v.ids, shape=(max(n, 1),))[:n].copy()
            max_fwd = v.max_fwd
        finally:
            lib().g2_view_free(C.byref(v))
        g = Graph(rp, ci, f"{self.name}+view")
        g.fwd_offsets = fo
        g.max_fwd = max_fwd
        return g, lsrc, ids

    def view_bins(self, max_bytes, radius=1, row_radius=None, min_root_degree=0, upper=False, forward=False,
                  ego=False):
        """(nbins, bin_of) from g2_view_bins: roots in id order, a bin closes when
        its view would exceed max_bytes."""
        bins = np.zeros(self.n, np.uint32)
        nb = C.c_uint32()
        rr = radius if row_radius is None else row_radius
        check(lib().g2_view_bins(_ptr(self.row_ptrs), _ptr(self.cols), self.n, radius, rr, min_root_degree,
                                 int(bool(upper)) | 4 * int(bool(forward)) | 8 * int(bool(ego)), int(max_bytes),
                                 _ptr(bins),
                                 C.byref(nb)), "g2_view_bins")
        return nb.value, bins

    def rebalance_bins(self, bin_of, nbins, devices=1, split_times=0, reorder=False):
        """(nbins, bin_of) after the reference's split / reorder of view bins
        (g2_view_bins_rebalance)."""
        bins = np.array(bin_of, dtype=np.uint32, copy=True)
        nb = C.c_uint32()
        check(lib().g2_view_bins_rebalance(_ptr(self.row_ptrs), self.n, _ptr(bins), nbins, devices, split_times,
                                           int(bool(reorder)), C.byref(nb)), "g2_view_bins_rebalance")
        return nb.value, bins

    # ----------------------------------------------------- degeneracy order
    def degeneracy_order(self):
        """(perm, core): perm[old] = new id (core shells ascending, degree
        ascending inside a shell), core[old] = core number."""
        perm = np.zeros(self.n, np.uint32)
        core = np.zeros(self.n, np.uint32)
        check(lib().g2_degeneracy_order(_ptr(self.row_ptrs), _ptr(self.cols), self.n, _ptr(perm), _ptr(core)),
              "g2_degeneracy_order")
        return perm, core

    def recode(self, perm):
        rp = np.zeros(self.n + 1, np.uint64)
        ci = np.zeros(self.m, np.uint32)
        check(lib().g2_recode(_ptr(self.row_ptrs), _ptr(self.cols), self.n, _ptr(np.ascontiguousarray(perm,
              dtype=np.uint32)), _ptr(rp), _ptr(ci)), "g2_recode")
        return Graph(rp, ci, self.name + "+recoded")

    def degeneracy_recoded(self):
        """The graph with ids in degeneracy order (what kmeans/kcore.cpp writes)."""
        perm, core = self.degeneracy_order()
        g = self.recode(perm)
        g.core = np.zeros(self.n, np.uint32)
        g.core[perm] = core
        return g

    # ------------------------------------------------ stream-byte models
    def _forward_degrees(self):
        rp = self.row_ptrs.astype(np.int64)
        src = np.repeat(np.arange(self.n, dtype=np.int64), np.diff(rp))
        fwd = self.cols.astype(np.int64) > src
        p = np.bincount(src[fwd], minlength=self.n).astype(np.int64)
        return src, fwd, p

    def clique_stream_bytes(self, k):
        """Bytes of the CSR the bitmap clique path must read once per root:
        the root's offsets and forward list, and for each forward neighbour its
        offsets and forward list (an upper bound: scans stop at the largest
        member of the root's forward list).  Roots with fewer than k-1 forward
        neighbours read their offsets only."""
        src, fwd, p = self._forward_degrees()
        s = np.bincount(src[fwd], weights=p[self.cols[fwd].astype(np.int64)], minlength=self.n)
        per = np.where(p >= k - 1, 20 + 24 * p + 4 * s, 20)
        return int(per.sum())

    def mce_stream_bytes(self):
        """Bytes of the CSR the MCE kernel must read once per root: offsets and
        neighbour list of the root, and offsets + forward list of every
        neighbour (rows of P0 and of the back neighbours)."""
        src, fwd, p = self._forward_degrees()
        deg = np.diff(self.row_ptrs.astype(np.int64))
        s = np.bincount(src, weights=p[self.cols.astype(np.int64)], minlength=self.n)
        per = np.where(p > 0, 20 + 24 * deg + 4 * s, 20)
        return int(per.sum())



def chung_lu_batch(count=64, seed=1, n_range=(10**3, 10**6), gamma_range=(2.1, 2.8), degree_range=(8.0, 40.0)):
    """A batch of Chung-Lu power-law graphs, degeneracy-ordered: n log-uniform
    in n_range, exponent uniform in gamma_range, average degree uniform in
    degree_range, one seed per graph (all drawn from `seed`)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        gamma = float(rng.uniform(*gamma_range))
        deg = float(rng.uniform(*degree_range))
        g = Graph.chung_lu(n, gamma, deg, seed=int(rng.integers(1, 2**31))).degeneracy_recoded()
        g.spec = {"n": n, "gamma": gamma, "avg_degree": deg}
        out.append(g)
    return out
