"""B200-native routing hot path: L-pattern costing, Boruvka RMST and the
Fenwick edge commit of SammithKanur/iitmGlobalRouter's -bit_pmodel router.

The compute lives in ``lib/libiitmgr_b200.so`` (hand-written sm_100a CUDA and
C++ host code behind the C ABI of ``include/iitmgr_b200.h``); this package is a
thin ctypes mirror used by tests, the benchmark and Python callers.
"""
from ._capi import GRError, LIB_PATH, lib  # noqa: F401
from .router import Design, Router, pair_count, slot_count  # noqa: F401

__all__ = ["Design", "Router", "GRError", "lib", "LIB_PATH", "pair_count", "slot_count"]
