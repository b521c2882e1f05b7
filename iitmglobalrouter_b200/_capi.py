"""ctypes bindings of include/iitmgr_b200.h.

The shared library is built in-tree (``python -m iitmglobalrouter_b200.build``)
and loaded from ``iitmglobalrouter_b200/lib``. There is no fallback: if the
library is missing, importing a routing entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libiitmgr_b200.so"

GR_OK = 0
ERRORS = {
    -1: "invalid argument", -2: "CUDA runtime error", -3: "out of memory", -4: "call out of order",
    -5: "net has more pins than supported", -6: "a kernel reported invalid data",
    -7: "file could not be read or written", -8: "malformed input text", -9: "capacity is not an integer",
}
GR_ST_BAD_EDGE, GR_ST_BAD_PATTERN, GR_ST_MST_ROUNDS, GR_ST_BAD_PIN = 0x1, 0x2, 0x4, 0x8
GR_PLAN_GRAPH = 0x1
GR_WRT_MERGE, GR_WRT_RSEG, GR_WRT_PPATCH = 0x1, 0x2, 0x4
GR_MAX_PINS = 4096
GR_STATIC_MAX_NETS, GR_STATIC_MAX_PINS = 65536, 1024
GR_PROF_KINDS = 10
GR_TUNE_MST_MID_THREADS, GR_TUNE_MST_BIG_THREADS, GR_TUNE_MST_CLUSTER_THREADS, GR_TUNE_MST_CLUSTER_MIN_PINS = 0, 1, 2, 3
GR_TUNE_LPAT_SPLIT = 4
GR_LA_DEMAND, GR_LA_EXCESS = 0, 1
GR_TUNE_MST_QUEUE = 5
GR_TUNE_PARAMS = 6

# every function of include/iitmgr_b200.h: name -> (restype, argtypes)
_P, _I, _I64, _U64, _D = C.c_void_p, C.c_int, C.c_int64, C.c_uint64, C.c_double
_PP = C.POINTER(C.c_void_p)
SIGNATURES = {
    "gr_version": (_I, []),
    "gr_error_string": (C.c_char_p, [_I]),
    "gr_create": (_I, [_PP, _I, _I, _I, _I, _P]),
    "gr_destroy": (_I, [_P]),
    "gr_reset": (_I, [_P, _P]),
    "gr_set_nets": (_I, [_P, C.c_int32, _P, _P]),
    "gr_lpattern": (_I, [_P, _P, _I64, _P, _P, _P]),
    "gr_brvsk_build": (_I, [_P, _P, C.c_int32, _P, _P, _P, _P]),
    "gr_brvsk_build_static": (_I, [_P, C.c_int32, _P, _P, _P, _P, _P]),
    "gr_mst_bit_commit": (_I, [_P, _P, C.c_int32, _P, _P, _P, _P]),
    "gr_route_batch": (_I, [_P, _P, C.c_int32, _P, _P, _P, _P, _P, _P]),
    "gr_plan_set": (_I, [_P, C.c_int32, _P, _P]),
    "gr_plan_slots": (_I64, [_P]),
    "gr_route_plan": (_I, [_P, C.c_int32, C.c_int32, _P, _P, _I, _P]),
    "gr_route_design_host": (_I, [_P, C.c_int32, _P, _P, C.c_int32, _P, _P, _P, _P, _I]),
    "gr_sync": (_I, [_P]),
    "gr_status": (C.c_uint32, [_P]),
    "gr_clear_status": (_I, [_P]),
    "gr_get_capr": (_I, [_P, _P]),
    "gr_get_demand": (_I, [_P, _P]),
    "gr_get_fenwick": (_I, [_P, _P]),
    "gr_stream": (_P, [_P]),
    "gr_launch_count": (_I64, [_P]),
    "gr_features": (_I, [_P, _P, C.c_float, _P]),
    "gr_set_lookahead": (_I, [_P, _P, C.c_float, _P]),
    "gr_tune_set": (_I, [_P, _I, _I]),
    "gr_tune_get": (_I, [_P, _I, _P]),
    "gr_profile_enable": (_I, [_P, _I]),
    "gr_profile_read": (_I, [_P, _P, _P, _I]),
    "gr_kernel_name": (C.c_char_p, [_I]),
    "gr_design_generate": (_I, [_PP, _I, _U64, _I64]),
    "gr_design_generate_custom": (_I, [_PP, _I, _I, _I, _I, _I, _D, _I, _I, _I64, _D, _I, _D, _D, _I, _U64]),
    "gr_design_read": (_I, [_PP, C.c_char_p, C.c_char_p, _I]),
    "gr_design_write": (_I, [_P, C.c_char_p, C.c_char_p]),
    "gr_design_free": (_I, [_P]),
    "gr_design_dims": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "gr_design_caps": (_I, [_P, _P]),
    "gr_design_nets": (_I, [_P, _P, _P]),
    "gr_design_net_name": (_I, [_P, C.c_int32, C.c_char_p, _I64]),
    "gr_design_batch": (_I, [_P, _I, _P, _P]),
    "gr_design_plan": (_I, [_P, _P, _P, _P, _P]),
    "gr_design_set_plan": (_I, [_P, C.c_int32, _P, _P]),
    "gr_design_write_routes": (_I, [_P, C.c_char_p, _P, _P, _I, _I, _P]),
    "gr_design_eval": (_I, [_P, _P, _P]),
    "gr_cnn_create": (_I, [_PP, _I, _I, _I, _I, _I, _I, _I, _U64]),
    "gr_cnn_destroy": (_I, [_P]),
    "gr_plan_check": (_I, [_P]),
    "gr_design_gather_bytes": (_I, [_P, _I, _P]),
    "gr_cnn_num_params": (_I64, [_P]),
    "gr_cnn_info": (_I, [_P, _P, _P, _P, _P, _P]),
    "gr_route_design_lookahead_host": (_I, [_P, _P, C.c_int32, C.c_float, _I, _P, _P]),
    "gr_cnn_get_params": (_I, [_P, _P]),
    "gr_cnn_set_params": (_I, [_P, _P]),
    "gr_cnn_forward": (_I, [_P, _P, _P]),
    "gr_cnn_forward_async": (_I, [_P, _P, _P, _P]),
    "gr_cnn_check": (_I, [_P]),
    "gr_route_plan_lookahead": (_I, [_P, _P, C.c_int32, C.c_float, _I, _P, _P, _I, _P]),
    "gr_cnn_grads": (_I, [_P, _P, _P, _P, _P]),
    "gr_cnn_train_step": (_I, [_P, _P, _P, C.c_float, _P]),
    "gr_cnn_gemm_test": (_I, [_I, _I, _I, _P, _P, _P, _I]),
}

_lib = None


class GRError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: {ERRORS.get(code, 'error')} ({code})" if what else ERRORS.get(code, str(code)))


def lib() -> C.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python -m iitmglobalrouter_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != GR_OK:
        raise GRError(rc, what)


def ptr(a) -> int | None:
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "array must be contiguous"
        return a.ctypes.data
    assert a.is_contiguous(), "tensor must be contiguous"
    return a.data_ptr()


def i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)
