"""g2aimd - B200-native subgraph search (maximal cliques and plan-driven
subgraph enumeration) behind the C ABI of include/g2_aimd.h.

Python is the test/bench harness and the reference-style host driver; all
enumeration runs in libg2aimd.so (hand-written sm_100a CUDA).
"""
from ._lib import G2Error, G2Opts, G2Plan, lib  # noqa: F401
from .graph import Graph  # noqa: F401
