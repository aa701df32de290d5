"""ctypes binding of libg2aimd.so (the C ABI declared in include/g2_aimd.h).

The library is built in-tree by g2-aimd_b200/build.py.  Loading fails loudly if
it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libg2aimd.so")

G2_MAX_QUERY = 8
Q = G2_MAX_QUERY
u32, u64, i32 = C.c_uint32, C.c_uint64, C.c_int
P = C.POINTER


class G2Plan(C.Structure):
    _fields_ = [
        ("k", u32), ("hop", u32), ("root_degree", u32),
        ("order", u32 * Q), ("id2order", u32 * Q),
        ("bn_count", u32 * Q), ("bn", (u32 * Q) * Q), ("parent", u32 * Q),
        ("cond_count", u32 * Q), ("cond", ((u32 * 2) * Q) * Q),
        ("share", u32 * Q),
        ("pre_bn_count", u32 * Q), ("pre_bn", (u32 * Q) * Q),
        ("pre_cond_count", u32 * Q), ("pre_cond", ((u32 * 2) * Q) * Q),
        ("after_bn_count", u32 * Q), ("after_bn", (u32 * Q) * Q),
        ("after_cond_count", u32 * Q), ("after_cond", ((u32 * 2) * Q) * Q),
        ("strategy", u32 * (Q + 1)), ("moving_lvl", u32 * Q),
    ]


class G2BatchGraph(C.Structure):
    _fields_ = [("row_ptrs", P(u64)), ("cols", P(u32)), ("n", u64), ("m", u64), ("core", P(u32))]


class G2Opts(C.Structure):
    _fields_ = [
        ("blocks", u32), ("warps_per_block", u32), ("schedule", u32),
        ("split_granularity", u32), ("scores", P(C.c_float)),
        ("root_nodes", P(u64)), ("work_bytes", P(u64)),
        ("intersect_mode", u32), ("flags", u32), ("split_depth", u32), ("root_cost", P(u64)),
        ("chunk", u32), ("spill_kcycles", u32), ("ctas_per_sm", u32), ("wait_cycles", u32),
        ("deadline_ms", u32),
    ]


class G2View(C.Structure):
    _fields_ = [("row_ptrs", P(u64)), ("cols", P(u32)), ("fwd_offsets", P(u32)), ("sources", P(u32)),
                ("ids", P(u32)), ("n", u64), ("m", u64), ("nsrc", u64), ("max_fwd", u32)]


class G2ViewOpts(C.Structure):
    _fields_ = [("producers", u32), ("radius", u32), ("row_radius", u32), ("flags", u32), ("slots", u32)]


class G2ViewStats(C.Structure):
    _fields_ = [("bins", u64), ("view_vertices", u64), ("view_edges", u64), ("h2d_bytes", u64),
                ("max_view_bytes", u64), ("build_ms", C.c_double), ("wait_ms", C.c_double),
                ("total_ms", C.c_double), ("copy_ms", C.c_double), ("run_ms", C.c_double)]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


G2_VIEW_NO_BIN = 0xFFFFFFFF
G2_VIEW_UPPER, G2_VIEW_NO_UPPER, G2_VIEW_FORWARD, G2_VIEW_EGO, G2_VIEW_DEVICE = 1, 2, 4, 8, 16

_lib = None


def lib():
    """Load and declare the library once (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python g2-aimd_b200/build.py`")
    L = C.CDLL(LIB_PATH)
    sig = {
        "g2_version": (C.c_char_p, []),
        "g2_strerror": (C.c_char_p, [i32]),
        "g2_last_cuda_error": (C.c_char_p, [C.c_void_p]),
        "g2_open": (i32, [i32, u64, P(C.c_void_p)]),
        "g2_close": (i32, [C.c_void_p]),
        "g2_load_csr": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u64, u64]),
        "g2_load_csr_device": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u64, u64]),
        "g2_set_plan": (i32, [C.c_void_p, P(G2Plan)]),
        "g2_mce_run": (i32, [C.c_void_p, C.c_void_p, u64, P(G2Opts), P(u64), C.c_void_p, u32]),
        "g2_match_run": (i32, [C.c_void_p, C.c_void_p, u64, P(G2Opts), P(u64)]),
        "g2_mce_run_device": (i32, [C.c_void_p, C.c_void_p, u64, P(G2Opts), C.c_void_p, u32, C.c_void_p]),
        "g2_match_run_device": (i32, [C.c_void_p, C.c_void_p, u64, P(G2Opts), C.c_void_p, C.c_void_p]),
        "g2_run_status": (i32, [C.c_void_p, C.c_void_p]),
        "g2_last_launch_count": (u64, [C.c_void_p]),
        "g2_pass_time_ms": (i32, [C.c_void_p, i32, P(C.c_float)]),
        "g2_last_work_bytes": (i32, [C.c_void_p, P(u64)]),
        "g2_last_spill_stats": (i32, [C.c_void_p, P(u64), P(u64)]),
        "g2_reserve": (i32, [C.c_void_p, u64]),
        "g2_set_host_spill": (i32, [C.c_void_p, u64]),
        "g2_degeneracy_order_device": (i32, [C.c_void_p, P(u32), P(u32)]),
        "g2_degeneracy_recode_device": (i32, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "g2_copy_csr": (i32, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "g2_batch_load": (i32, [C.c_void_p, C.c_void_p, u32]),
        "g2_batch_mce": (i32, [C.c_void_p, C.c_void_p, P(u64), P(u64), u32]),
        "g2_batch_match": (i32, [C.c_void_p, C.c_void_p, P(u64)]),
        "g2_view_mce": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u64, C.c_void_p, u32, P(G2ViewOpts), P(G2Opts),
                              P(u64), C.c_void_p, u32, C.c_void_p, P(G2ViewStats)]),
        "g2_view_match": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u64, C.c_void_p, u32, P(G2ViewOpts),
                                P(G2Opts), P(u64), C.c_void_p, P(G2ViewStats)]),
        "g2_view_materialize": (i32, [C.c_void_p, C.c_void_p, u64, C.c_void_p, u64, u32, u32, u32, u32,
                                      P(G2View)]),
        "g2_view_free": (None, [P(G2View)]),
        "g2_view_materialize_device": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u64, C.c_void_p, u64, u32, u32,
                                             P(G2View)]),
        "g2_plan_view_radius": (i32, [P(G2Plan), P(u32), P(u32), P(u32), P(u32)]),
        "g2_view_bins": (i32, [C.c_void_p, C.c_void_p, u64, u32, u32, u32, u32, u64, C.c_void_p, P(u32)]),
        "g2_view_bins_rebalance": (i32, [C.c_void_p, u64, C.c_void_p, u32, u32, u32, i32, P(u32)]),
        "g2_shell_bins": (i32, [C.c_void_p, u64, u32, C.c_void_p]),
        "g2_load_core": (i32, [C.c_void_p, C.c_void_p]),
        "g2_root_features": (i32, [C.c_void_p, C.c_void_p, u64, C.c_void_p]),
        "g2_model_train": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u64, u32, u32, C.c_float, u64, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
        "g2_model_grad": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u32, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p]),
        "g2_model_predict": (i32, [C.c_void_p, C.c_void_p, u64, C.c_void_p, C.c_void_p, C.c_void_p]),
        "g2_set_model": (i32, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "g2_match_count_noalloc": (i32, [C.c_void_p, C.c_void_p, u64, u64, C.c_void_p, C.c_void_p, C.c_void_p]),
        "g2_plan_preset": (i32, [i32, P(G2Plan)]),
        "g2_plan_build": (i32, [u32, C.c_void_p, u32, P(G2Plan)]),
        "g2_read_bin": (i32, [C.c_char_p, P(C.c_void_p), P(C.c_void_p), P(u64), P(u64)]),
        "g2_write_bin": (i32, [C.c_char_p, C.c_void_p, C.c_void_p, u64, u64]),
        "g2_free": (None, [C.c_void_p]),
        "g2_read_snap": (i32, [C.c_char_p, i32, P(C.c_void_p), P(C.c_void_p), P(u64), P(u64)]),
        "g2_write_vbmap": (i32, [C.c_char_p, u32, C.c_void_p, u64]),
        "g2_read_vbmap": (i32, [C.c_char_p, u64, P(u32), C.c_void_p]),
        "g2_degeneracy_order": (i32, [C.c_void_p, C.c_void_p, u64, C.c_void_p, C.c_void_p]),
        "g2_recode": (i32, [C.c_void_p, C.c_void_p, u64, C.c_void_p, C.c_void_p, C.c_void_p]),
        "g2_gen_er": (i32, [u64, C.c_double, u32, u32, u64, P(C.c_void_p), P(C.c_void_p), P(u64), P(u64)]),
        "g2_gen_rmat": (i32, [u32, u32, C.c_double, C.c_double, C.c_double, u32, u32, u32, u64,
                              P(C.c_void_p), P(C.c_void_p), P(u64), P(u64)]),
        "g2_gen_rmat_device": (i32, [C.c_void_p, u32, u32, C.c_double, C.c_double, C.c_double, u32, u32, u32,
                                     u64, P(u64)]),
        "g2_gen_chunglu": (i32, [u64, C.c_double, C.c_double, u64, P(C.c_void_p), P(C.c_void_p),
                                 P(u64), P(u64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class G2Error(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        msg = lib().g2_strerror(code).decode()
        super().__init__(f"{where}: {msg} ({code})" if where else f"{msg} ({code})")


def check(code, where=""):
    if code != 0:
        raise G2Error(code, where)
    return code
