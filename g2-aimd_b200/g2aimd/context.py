"""Python side of the C ABI: a device context, query plans, and the two
enumerations (maximal cliques, plan-driven subgraph counts).

This mirrors the reference's app plugin surface: `Context.mce` is what
Worker<BKExpandSequential> computes (sum of the "Total No. of Cliques:" lines,
app_BK/BK.h:72-76) and `Context.match` is Worker<GMatchApp>'s "Total counts:"
(system/worker.h:273-279).  All work runs in libg2aimd.so on the GPU; errors
are raised, never hidden.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import G2_MAX_QUERY, G2Opts, G2Plan, check, lib

SCHED = {"given": 0, "heuristic": 1, "scores": 2, "learned": 3}
FLAG_TIME_KERNELS, FLAG_WORK_MODEL, FLAG_SPLIT, FLAG_NO_SPLIT, FLAG_NO_SPILL, FLAG_L2_PERSIST = 1, 2, 4, 8, 16, 32
MODEL_FEATURES, MODEL_PARAMS, MODEL_NORM = 8, 4801, 18


class Plan:
    """A query plan (GMContext arrays, system/appbase.h:11-68)."""

    def __init__(self, raw: G2Plan):
        self.raw = raw

    @staticmethod
    def preset(query_id: int) -> "Plan":
        p = G2Plan()
        check(lib().g2_plan_preset(int(query_id), C.byref(p)), f"plan preset {query_id}")
        return Plan(p)

    @staticmethod
    def from_edges(k: int, edges) -> "Plan":
        e = np.ascontiguousarray(np.asarray(edges, dtype=np.uint32).reshape(-1, 2))
        p = G2Plan()
        check(lib().g2_plan_build(k, e.ctypes.data_as(C.c_void_p), e.shape[0], C.byref(p)), "plan build")
        return Plan(p)

    @property
    def k(self) -> int:
        return self.raw.k

    def view_shape(self):
        """dict(radius, row_radius, min_root_degree, upper, forward): the view this plan's
        roots need (g2_plan_view_radius); keyword arguments of Graph.view."""
        r, rr, d, f = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib().g2_plan_view_radius(C.byref(self.raw), C.byref(r), C.byref(rr), C.byref(d), C.byref(f)),
              "g2_plan_view_radius")
        return {"radius": r.value, "row_radius": rr.value, "min_root_degree": d.value, "upper": bool(f.value & 1),
                "forward": bool(f.value & 4)}

    def to_dict(self) -> dict:
        """Same field layout as the reference-planner fixtures."""
        r, k = self.raw, self.raw.k
        lst = lambda cnt, arr: [[arr[i][j] for j in range(cnt[i])] for i in range(k)]  # noqa: E731
        lst2 = lambda cnt, arr: [[[arr[i][j][0], arr[i][j][1]] for j in range(cnt[i])] for i in range(k)]  # noqa
        return {
            "k": k, "hop": r.hop, "root_degree": r.root_degree,
            "order": list(r.order[:k]), "id2order": list(r.id2order[:k]),
            "bn_count": list(r.bn_count[:k]), "bn": lst(r.bn_count, r.bn), "share": list(r.share[:k]),
            "pre_bn": lst(r.pre_bn_count, r.pre_bn), "after_bn": lst(r.after_bn_count, r.after_bn),
            "cond": lst2(r.cond_count, r.cond), "pre_cond": lst2(r.pre_cond_count, r.pre_cond),
            "after_cond": lst2(r.after_cond_count, r.after_cond),
            "strategy": list(r.strategy[:k + 1]), "moving_lvl": list(r.moving_lvl[:k]),
        }

    def flat(self):
        """(order, id2order, bn_count, bn[k*k], cond_count, cond[k*k*2]) with
        the reference's strides, for the oracle."""
        r, k = self.raw, self.raw.k
        bn = np.zeros(k * k, np.uint32)
        cond = np.zeros(k * k * 2, np.uint32)
        for i in range(k):
            for j in range(r.bn_count[i]):
                bn[i * k + j] = r.bn[i][j]
            for j in range(r.cond_count[i]):
                cond[(i * k + j) * 2] = r.cond[i][j][0]
                cond[(i * k + j) * 2 + 1] = r.cond[i][j][1]
        return (np.array(r.order[:k], np.uint32), np.array(r.id2order[:k], np.uint32),
                np.array(r.bn_count[:k], np.uint32), bn, np.array(r.cond_count[:k], np.uint32), cond)


def _opts(warps_per_block=0, blocks=0, schedule="given", scores=None, root_nodes=None, intersect_mode=0,
          granularity=0, chunk=0, flags=0, work_bytes=None, root_cost=None, split=False, split_depth=0,
          spill_kcycles=0, ctas_per_sm=0, wait_cycles=0, deadline_ms=0):
    o = G2Opts()
    o.deadline_ms = deadline_ms
    o.wait_cycles = wait_cycles
    o.ctas_per_sm = ctas_per_sm
    o.split_depth = split_depth
    o.spill_kcycles = spill_kcycles
    o.flags = flags | (FLAG_SPLIT if split else 0)
    o.chunk = chunk
    o.warps_per_block = warps_per_block
    o.blocks = blocks
    o.schedule = SCHED[schedule]
    o.split_granularity = granularity
    o.intersect_mode = intersect_mode
    keep = []
    if scores is not None:
        s = np.ascontiguousarray(scores, dtype=np.float32)
        keep.append(s)
        o.scores = s.ctypes.data_as(C.POINTER(C.c_float))
    if root_nodes is not None:
        o.root_nodes = root_nodes.ctypes.data_as(C.POINTER(C.c_uint64))
    if work_bytes is not None:
        o.work_bytes = work_bytes.ctypes.data_as(C.POINTER(C.c_uint64))
    if root_cost is not None:
        o.root_cost = root_cost.ctypes.data_as(C.POINTER(C.c_uint64))
    return o, keep


G2_ERR_DEADLINE = -11


class Context:
    """One device context (g2_open).  Load a graph, then run enumerations."""

    def __init__(self, device: int = 0, scratch_bytes: int = 0):
        self._h = C.c_void_p()
        check(lib().g2_open(device, scratch_bytes, C.byref(self._h)), "g2_open")
        self.graph = None
        self.n = 0
        self.expired = False  # the last MCE run's time budget (deadline_ms) ran out

    def close(self):
        if self._h:
            check(lib().g2_close(self._h), "g2_close")
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def cuda_error(self) -> str:
        return lib().g2_last_cuda_error(self._h).decode()

    def launches(self) -> int:
        return int(lib().g2_last_launch_count(self._h))

    def batch_load(self, graphs):
        """Load several graphs as one disjoint union (g2_batch_load); cores are
        loaded too when every graph has them (degeneracy_recoded graphs do)."""
        from ._lib import G2BatchGraph
        arr = (G2BatchGraph * len(graphs))()
        keep = []
        for i, g in enumerate(graphs):
            rp = np.ascontiguousarray(g.row_ptrs, dtype=np.uint64)
            ci = np.ascontiguousarray(g.cols, dtype=np.uint32)
            core = getattr(g, "core", None)
            keep += [rp, ci]
            arr[i].row_ptrs = rp.ctypes.data_as(C.POINTER(C.c_uint64))
            arr[i].cols = ci.ctypes.data_as(C.POINTER(C.c_uint32))
            arr[i].n, arr[i].m = g.n, g.m
            if core is not None:
                core = np.ascontiguousarray(core, dtype=np.uint32)
                keep.append(core)
                arr[i].core = core.ctypes.data_as(C.POINTER(C.c_uint32))
        self._check(lib().g2_batch_load(self._h, arr, len(graphs)), "g2_batch_load")
        self.graph = None
        self.n = int(sum(g.n for g in graphs))
        self.batch = len(graphs)
        del keep
        return self

    def batch_mce(self, hist_len=256, **kw):
        """(maximal cliques per graph, size histogram of all) of the loaded batch."""
        o, keep = _opts(**kw)
        counts = np.zeros(self.batch, np.uint64)
        hist = np.zeros(hist_len, np.uint64)
        self._check(lib().g2_batch_mce(self._h, C.byref(o), counts.ctypes.data_as(C.POINTER(C.c_uint64)),
                                       hist.ctypes.data_as(C.POINTER(C.c_uint64)), hist_len), "g2_batch_mce")
        del keep
        return counts, hist

    def batch_match(self, plan: Plan = None, **kw):
        """Matches per graph of the loaded batch."""
        if plan is not None:
            self.set_plan(plan)
        o, keep = _opts(**kw)
        counts = np.zeros(self.batch, np.uint64)
        self._check(lib().g2_batch_match(self._h, C.byref(o), counts.ctypes.data_as(C.POINTER(C.c_uint64))),
                    "g2_batch_match")
        del keep
        return counts

    def degeneracy_order(self):
        """(perm, core) of the loaded graph computed on the device."""
        perm = np.zeros(self.n, np.uint32)
        core = np.zeros(self.n, np.uint32)
        self._check(lib().g2_degeneracy_order_device(self._h, perm.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                     core.ctypes.data_as(C.POINTER(C.c_uint32))),
                    "g2_degeneracy_order_device")
        return perm, core

    def degeneracy_recode(self):
        """Rename the loaded graph by its degeneracy order on the device
        (g2_degeneracy_recode_device); core numbers are loaded under the new
        names.  Returns (perm, core) by old id."""
        perm = np.zeros(self.n, np.uint32)
        core = np.zeros(self.n, np.uint32)
        self._check(lib().g2_degeneracy_recode_device(self._h, perm.ctypes.data_as(C.c_void_p),
                                                      core.ctypes.data_as(C.c_void_p)),
                    "g2_degeneracy_recode_device")
        self.graph = None
        return perm, core

    def copy_csr(self, m: int):
        """The loaded CSR copied back to host memory (m column entries)."""
        from .graph import Graph
        rp = np.zeros(self.n + 1, np.uint64)
        ci = np.zeros(max(m, 1), np.uint32)
        self._check(lib().g2_copy_csr(self._h, rp.ctypes.data_as(C.c_void_p), ci.ctypes.data_as(C.c_void_p)),
                    "g2_copy_csr")
        return Graph(rp, ci[:m].copy())

    def set_host_spill(self, nbytes: int):
        """Managed spill slab for MCE roots no scratch slab holds (0: none)."""
        self._check(lib().g2_set_host_spill(self._h, nbytes), "g2_set_host_spill")
        return self

    def reserve(self, max_sources: int = 0):
        """Allocate the run buffers now (g2_reserve) instead of in the first run."""
        self._check(lib().g2_reserve(self._h, max_sources), "g2_reserve")
        return self

    def spill_stats(self):
        """(records, pool bytes) the last MCE run handed from long walks to idle warps."""
        r, b = C.c_uint64(), C.c_uint64()
        self._check(lib().g2_last_spill_stats(self._h, C.byref(r), C.byref(b)), "g2_last_spill_stats")
        return r.value, b.value

    def pass_times(self):
        """Device ms of the last run's passes (after a run with flags=1): three
        for MCE (main, two deferred), one for a match run."""
        out = []
        for k in range(3):
            ms = C.c_float()
            rc = lib().g2_pass_time_ms(self._h, k, C.byref(ms))
            if rc == -1 and k > 0:
                break
            self._check(rc, "g2_pass_time_ms")
            out.append(ms.value)
        return out

    def _check(self, rc, where):
        if rc != 0:
            err = self.cuda_error()
            check(rc, where + (f" [{err}]" if err else ""))

    def load(self, graph):
        self._check(lib().g2_load_csr(self._h, graph.row_ptrs.ctypes.data_as(C.c_void_p),
                                      graph.cols.ctypes.data_as(C.c_void_p), graph.n, graph.m), "g2_load_csr")
        self.graph = graph
        self.n = graph.n
        return self

    def load_device(self, d_row_ptrs: int, d_cols: int, n: int, m: int):
        """Borrow a CSR already in device memory (raw device pointers)."""
        self._check(lib().g2_load_csr_device(self._h, C.c_void_p(d_row_ptrs), C.c_void_p(d_cols), n, m),
                    "g2_load_csr_device")
        self.graph = None
        self.n = n
        return self

    def gen_rmat(self, scale, edge_factor, a=0.57, b=0.19, c=0.19, planted=0, pmin=0, pmax=0, seed=1):
        """Build Graph.rmat(...)'s graph on the device as this context's graph
        (g2_gen_rmat_device); returns its directed entry count m."""
        m = C.c_uint64()
        self._check(lib().g2_gen_rmat_device(self._h, scale, edge_factor, a, b, c, planted, pmin, pmax, seed,
                                             C.byref(m)), "g2_gen_rmat_device")
        self.graph, self.n, self.m = None, 1 << scale, m.value
        return m.value

    def view_device(self, graph, sources, min_root_degree=0, upper=False, forward=False):
        """Graph.view's radius-1 view of `sources` built by this context's GPU
        (g2_view_materialize_device): (view graph, local sources, global ids).
        Releases the context's loaded graph."""
        from ._lib import G2View
        from .graph import Graph
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        v = G2View()
        self._check(lib().g2_view_materialize_device(
            self._h, graph.row_ptrs.ctypes.data_as(C.c_void_p), graph.cols.ctypes.data_as(C.c_void_p), graph.n,
            src.ctypes.data_as(C.c_void_p), src.size, min_root_degree,
            int(bool(upper)) | 4 * int(bool(forward)), C.byref(v)), "g2_view_materialize_device")
        self.graph, self.n = None, 0
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
        g = Graph(rp, ci, f"{graph.name}+view")
        g.fwd_offsets = fo
        g.max_fwd = max_fwd
        return g, lsrc, ids

    def set_plan(self, plan: Plan):
        self._check(lib().g2_set_plan(self._h, C.byref(plan.raw)), "g2_set_plan")
        return self

    def mce(self, sources=None, hist_len=256, root_nodes=False, root_cost=None, **kw):
        """(count, hist) of maximal cliques rooted at `sources` (default: all);
        with root_nodes=True also the search-tree node count per source.  A
        uint64 array passed as root_cost receives SM cycles per source."""
        src = None if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
        nsrc = 0 if src is None else src.size
        rn = np.zeros(nsrc if src is not None else self.n, np.uint64) if root_nodes else None
        o, keep = _opts(root_nodes=rn, root_cost=root_cost, **kw)
        count = C.c_uint64()
        hist = np.zeros(hist_len, np.uint64)
        rc = lib().g2_mce_run(self._h, None if src is None else src.ctypes.data_as(C.c_void_p), nsrc,
                              C.byref(o), C.byref(count), hist.ctypes.data_as(C.c_void_p), hist_len)
        # with a time budget (deadline_ms), G2_ERR_DEADLINE is a result: the
        # outputs hold the roots that finished (root_nodes > 0)
        self.expired = rc == G2_ERR_DEADLINE and o.deadline_ms != 0
        if not self.expired:
            self._check(rc, "g2_mce_run")
        del keep
        return (count.value, hist, rn) if root_nodes else (count.value, hist)

    def match(self, plan: Plan = None, sources=None, root_counts=None, root_cost=None, **kw):
        """Embeddings admitted by the plan, rooted at `sources` (default: all).
        Optional uint64 arrays: root_counts (embeddings per source), root_cost
        (SM cycles per source)."""
        if plan is not None:
            self.set_plan(plan)
        src = None if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
        o, keep = _opts(root_nodes=root_counts, root_cost=root_cost, **kw)
        count = C.c_uint64()
        rc = lib().g2_match_run(self._h, None if src is None else src.ctypes.data_as(C.c_void_p),
                                0 if src is None else src.size, C.byref(o), C.byref(count))
        # with a time budget (deadline_ms), G2_ERR_DEADLINE is a result: the count
        # covers the roots that finished (root_cost > 0)
        self.expired = rc == G2_ERR_DEADLINE and o.deadline_ms != 0
        if not self.expired:
            self._check(rc, "g2_match_run")
        del keep
        return count.value

    # out-of-core runs over view bins: the graph stays in host memory
    def _view_args(self, graph, bin_of, nbins, producers, radius, row_radius, no_upper, ego=False, slots=0,
                   device=False):
        from ._lib import G2_VIEW_DEVICE, G2_VIEW_EGO, G2_VIEW_NO_UPPER, G2ViewOpts
        bins = np.ascontiguousarray(bin_of, dtype=np.uint32)
        if nbins is None:
            valid = bins[bins != 0xFFFFFFFF]
            nbins = int(valid.max()) + 1 if valid.size else 0
        vo = G2ViewOpts(producers, radius, row_radius,
                        (G2_VIEW_NO_UPPER if no_upper else 0) | (G2_VIEW_EGO if ego else 0) |
                        (G2_VIEW_DEVICE if device else 0), slots)
        return bins, nbins, vo

    def view_mce(self, graph, bin_of, nbins=None, hist_len=256, producers=0, radius=0, row_radius=0, ego=False,
                 slots=0, device=False, **kw):
        """(count, hist, per-bin counts, stats) of maximal cliques of a host graph
        enumerated view bin by view bin (g2_view_mce); ego: ego-network rows;
        device: views built by the GPU (G2_VIEW_DEVICE)."""
        from ._lib import G2ViewStats
        bins, nbins, vo = self._view_args(graph, bin_of, nbins, producers, radius, row_radius, False, ego, slots,
                                          device)
        o, keep = _opts(**kw)
        count = C.c_uint64()
        hist = np.zeros(hist_len, np.uint64)
        per_bin = np.zeros(max(nbins, 1), np.uint64)
        st = G2ViewStats()
        self._check(lib().g2_view_mce(self._h, graph.row_ptrs.ctypes.data_as(C.c_void_p),
                                      graph.cols.ctypes.data_as(C.c_void_p), graph.n,
                                      bins.ctypes.data_as(C.c_void_p), nbins, C.byref(vo), C.byref(o),
                                      C.byref(count), hist.ctypes.data_as(C.c_void_p), hist_len,
                                      per_bin.ctypes.data_as(C.c_void_p), C.byref(st)), "g2_view_mce")
        del keep
        self.graph, self.n = None, 0
        return count.value, hist, per_bin[:nbins], st.to_dict()

    def view_match(self, graph, bin_of, plan: Plan = None, nbins=None, producers=0, radius=0, row_radius=0,
                   no_upper=False, ego=False, slots=0, device=False, **kw):
        """(count, per-bin counts, stats) of the plan's matches in a host graph,
        view bin by view bin (g2_view_match)."""
        from ._lib import G2ViewStats
        if plan is not None:
            self.set_plan(plan)
        bins, nbins, vo = self._view_args(graph, bin_of, nbins, producers, radius, row_radius, no_upper, ego, slots,
                                          device)
        o, keep = _opts(**kw)
        count = C.c_uint64()
        per_bin = np.zeros(max(nbins, 1), np.uint64)
        st = G2ViewStats()
        self._check(lib().g2_view_match(self._h, graph.row_ptrs.ctypes.data_as(C.c_void_p),
                                        graph.cols.ctypes.data_as(C.c_void_p), graph.n,
                                        bins.ctypes.data_as(C.c_void_p), nbins, C.byref(vo), C.byref(o),
                                        C.byref(count), per_bin.ctypes.data_as(C.c_void_p), C.byref(st)),
                    "g2_view_match")
        del keep
        self.graph, self.n = None, 0
        return count.value, per_bin[:nbins], st.to_dict()

    # device-resident entry points (timing): pointers are raw device addresses
    def mce_device(self, d_out: int, hist_len: int, d_sources: int = 0, nsrc: int = 0, stream: int = 0, **kw):
        o, keep = _opts(**kw)
        self._check(lib().g2_mce_run_device(self._h, C.c_void_p(d_sources) if d_sources else None, nsrc,
                                            C.byref(o), C.c_void_p(d_out), hist_len, C.c_void_p(stream)),
                    "g2_mce_run_device")

    def match_device(self, d_out: int, d_sources: int = 0, nsrc: int = 0, stream: int = 0, **kw):
        o, keep = _opts(**kw)
        self._check(lib().g2_match_run_device(self._h, C.c_void_p(d_sources) if d_sources else None, nsrc,
                                              C.byref(o), C.c_void_p(d_out), C.c_void_p(stream)),
                    "g2_match_run_device")

    def run_status(self, stream: int = 0) -> int:
        """Outcome code of the last device-stream run on `stream` (g2_run_status;
        waits for the stream): 0, or the G2_ERR_* the synchronous entry point
        would have returned."""
        return lib().g2_run_status(self._h, C.c_void_p(stream))

    # ------------------------------------------------------ cost model
    def load_core(self, core):
        c = np.ascontiguousarray(core, dtype=np.uint32)
        self._check(lib().g2_load_core(self._h, c.ctypes.data_as(C.c_void_p)), "g2_load_core")

    def root_features(self, sources=None):
        src = None if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
        n = self.n if src is None else src.size
        out = np.zeros((n, MODEL_FEATURES), np.float32)
        self._check(lib().g2_root_features(self._h, None if src is None else src.ctypes.data_as(C.c_void_p),
                                           0 if src is None else src.size, out.ctypes.data_as(C.c_void_p)),
                    "g2_root_features")
        return out

    def set_model(self, model: "CostModel"):
        self._check(lib().g2_set_model(self._h, model.params.ctypes.data_as(C.c_void_p),
                                       model.norm.ctypes.data_as(C.c_void_p)), "g2_set_model")


class CostModel:
    """The learned root-cost model: 8 features -> 64 -> 64 -> 1, trained and
    evaluated by the library's tensor-core kernels (g2_model_*)."""

    def __init__(self, params, norm):
        self.params = np.ascontiguousarray(params, dtype=np.float32)
        self.norm = np.ascontiguousarray(norm, dtype=np.float32)
        assert self.params.size == MODEL_PARAMS and self.norm.size == MODEL_NORM

    @staticmethod
    def train(ctx: Context, X, cost, epochs=30, batch=1024, lr=3e-3, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        cost = np.ascontiguousarray(cost, dtype=np.float32)
        params = np.zeros(MODEL_PARAMS, np.float32)
        norm = np.zeros(MODEL_NORM, np.float32)
        losses = np.zeros(epochs, np.float32)
        ctx._check(lib().g2_model_train(ctx.handle, X.ctypes.data_as(C.c_void_p), cost.ctypes.data_as(C.c_void_p),
                                        X.shape[0], epochs, batch, lr, seed, params.ctypes.data_as(C.c_void_p),
                                        norm.ctypes.data_as(C.c_void_p), losses.ctypes.data_as(C.c_void_p)),
                   "g2_model_train")
        m = CostModel(params, norm)
        m.losses = losses
        return m

    def predict(self, ctx: Context, X):
        """Normalised log-cost predictions of feature rows X (n x 8)."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros(X.shape[0], np.float32)
        ctx._check(lib().g2_model_predict(ctx.handle, X.ctypes.data_as(C.c_void_p), X.shape[0],
                                          self.norm.ctypes.data_as(C.c_void_p),
                                          self.params.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)),
                   "g2_model_predict")
        return out

    def grad(self, ctx: Context, X, y):
        """(gradient of the mean squared error w.r.t. the parameters, loss) for
        normalised targets y, computed by the training kernel."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(MODEL_PARAMS, np.float32)
        loss = C.c_float()
        ctx._check(lib().g2_model_grad(ctx.handle, X.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p),
                                       X.shape[0], self.norm.ctypes.data_as(C.c_void_p),
                                       self.params.ctypes.data_as(C.c_void_p), g.ctypes.data_as(C.c_void_p),
                                       C.byref(loss)), "g2_model_grad")
        return g, loss.value

    def save(self, path):
        np.savez(path, params=self.params, norm=self.norm)

    @staticmethod
    def load(path):
        d = np.load(path)
        return CostModel(d["params"], d["norm"])


__all__ = ["Context", "Plan", "CostModel", "G2_MAX_QUERY"]
