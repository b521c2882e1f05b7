"""CPU oracle for the routing hot path -- TEST INFRASTRUCTURE ONLY.

A ctypes wrapper over oracle/gr_oracle.c, the plain-C restatement of the
reference's -bit_pmodel path (see gr_oracle.h for citations and the fixed
tie-break rules). Parity status: parity unpinned -- the reference has no
golden vectors and cannot be built here (it needs Boost); the oracle is
pinned by the hand-derived known-answer cases under tests/golden.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this module.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import build as _build

_P, _I, _I32, _I64 = C.c_void_p, C.c_int, C.c_int32, C.c_int64
_SIG = {
    "gro_enc": (C.c_int32, [_P, _I, _I, _I]),
    "gro_cost_of": (C.c_float, [_I]),
    "gro_cost_inc": (C.c_float, [_I]),
    "gro_grid_new": (_P, [_I, _I, _I, _P]),
    "gro_grid_free": (None, [_P]),
    "gro_grid_reset": (None, [_P]),
    "gro_query": (C.c_float, [_P, _I, _I, _I]),
    "gro_pattern_cost": (_I, [_P, C.c_int32, C.c_int32, _I, C.POINTER(C.c_float)]),
    "gro_lpattern_pair": (None, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_int16)]),
    "gro_lpattern": (None, [_P, _P, _I64, _P, _P, _I]),
    "gro_batch_pairs": (_I64, [_P, _P, _P, _I32, _P]),
    "gro_brvsk_net": (_I, [_I, _P, _I64, _P, _P]),
    "gro_brvsk_build": (_I, [_P, _P, _I32, _P, _P, _P, _I]),
    "gro_commit": (_I, [_P, _P, _P, _P, _I32, _P, _P, _P]),
    "gro_route_batch": (_I, [_P, _P, _P, _P, _I32, _P, _P, _P, _P, _P, _I]),
    "gro_route_batches": (_I, [_P, _P, _P, _P, _P, _I32, _P, _P, _I]),
    "gro_count_oob_pairs": (None, [_P, _P, _P, _P, _I32, _P]),
    "gro_lpattern_top2": (None, [_P, _P, _I64, _P, _P, _P, _I]),
}
_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(_build.build()))
        for k, (r, a) in _SIG.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


class _GridStruct(C.Structure):
    _fields_ = [("X", C.c_int), ("Y", C.c_int), ("Z", C.c_int), ("csize", C.c_int64),
                ("cap0", C.POINTER(C.c_int32)), ("capr", C.POINTER(C.c_int32)), ("fen", C.POINTER(C.c_float))]


def _p(a):
    return None if a is None else a.ctypes.data


def cost_of(c: int) -> float:
    return float(lib().gro_cost_of(c))


class Grid:
    """Grid state (capacities, remaining capacity, Fenwick nodes) on the CPU."""

    def __init__(self, X, Y, Z, cap):
        self.X, self.Y, self.Z = X, Y, Z
        self.csize = X * Y * Z
        cap = np.ascontiguousarray(cap, dtype=np.int32)
        assert cap.size == self.csize
        self._h = lib().gro_grid_new(X, Y, Z, _p(cap))
        if not self._h:
            raise MemoryError("gro_grid_new")
        self._s = C.cast(self._h, C.POINTER(_GridStruct)).contents

    def __del__(self):
        if getattr(self, "_h", None):
            lib().gro_grid_free(self._h)
            self._h = None

    def reset(self):
        lib().gro_grid_reset(self._h)

    def enc(self, z, x, y) -> int:
        return int(lib().gro_enc(self._h, z, x, y))

    def query(self, z, x, y) -> float:
        return float(lib().gro_query(self._h, z, x, y))

    def capr(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._s.capr, shape=(self.csize,)).copy()

    def demand(self) -> np.ndarray:
        cap0 = np.ctypeslib.as_array(self._s.cap0, shape=(self.csize,))
        return (cap0 - self.capr()).astype(np.int32)

    def fenwick(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._s.fen, shape=(self.csize,)).copy()

    def pattern_cost(self, e1, e2, cpat):
        c = C.c_float()
        ok = lib().gro_pattern_cost(self._h, e1, e2, cpat, C.byref(c))
        return (float(c.value) if ok else None)

    def lpattern(self, pairs, nthreads=1):
        pairs = np.ascontiguousarray(pairs, dtype=np.int32)
        n = pairs.size // 2
        cost = np.empty(n, dtype=np.float32)
        pat = np.empty(n, dtype=np.int16)
        lib().gro_lpattern(self._h, _p(pairs), n, _p(cost), _p(pat), nthreads)
        return cost, pat

    def lpattern_top2(self, pairs, nthreads=1):
        """(cost, pattern, cheapest cost among the other valid patterns)."""
        pairs = np.ascontiguousarray(pairs, dtype=np.int32)
        n = pairs.size // 2
        cost = np.empty(n, dtype=np.float32)
        pat = np.empty(n, dtype=np.int16)
        cost2 = np.empty(n, dtype=np.float32)
        lib().gro_lpattern_top2(self._h, _p(pairs), n, _p(cost), _p(pat), _p(cost2), nthreads)
        return cost, pat, cost2

    def set_state(self, capr, fen):
        """Overwrites the remaining capacities and the Fenwick nodes (a cost
        state recorded elsewhere, e.g. by the reference's own code)."""
        np.ctypeslib.as_array(self._s.capr, shape=(self.csize,))[:] = np.asarray(capr, dtype=np.int32)
        np.ctypeslib.as_array(self._s.fen, shape=(self.csize,))[:] = np.asarray(fen, dtype=np.float32)

    def commit(self, pin_ofs, pins, net_ids, mst, pair_pat):
        pin_ofs = np.ascontiguousarray(pin_ofs, dtype=np.int64)
        pins = np.ascontiguousarray(pins, dtype=np.int32)
        ids = np.ascontiguousarray(net_ids, dtype=np.int32)
        mst = np.ascontiguousarray(mst, dtype=np.int64)
        pp = np.ascontiguousarray(pair_pat, dtype=np.int16)
        mst_pat = np.empty(mst.size, dtype=np.int32)
        rc = lib().gro_commit(self._h, _p(pin_ofs), _p(pins), _p(ids), len(ids), _p(mst), _p(pp), _p(mst_pat))
        return rc, mst_pat

    def route_batch(self, pin_ofs, pins, net_ids, nthreads=1):
        """One batch; returns dict(pair_cost, pair_pat, mst, mst_pat, dist, rc)."""
        pin_ofs = np.ascontiguousarray(pin_ofs, dtype=np.int64)
        pins = np.ascontiguousarray(pins, dtype=np.int32)
        ids = np.ascontiguousarray(net_ids, dtype=np.int32)
        n = (pin_ofs[ids + 1] - pin_ofs[ids]).astype(np.int64)
        P = int((n * (n - 1) // 2).sum())
        M = int(n.sum())
        pc = np.empty(max(P, 1), dtype=np.float32)
        pp = np.empty(max(P, 1), dtype=np.int16)
        mst = np.empty(max(M, 1), dtype=np.int64)
        mp = np.empty(max(M, 1), dtype=np.int32)
        dist = np.empty(max(len(ids), 1), dtype=np.float32)
        rc = lib().gro_route_batch(self._h, _p(pin_ofs), _p(pins), _p(ids), len(ids), _p(pc), _p(pp), _p(mst),
                                   _p(mp), _p(dist), nthreads)
        return dict(rc=rc, pair_cost=pc[:P], pair_pat=pp[:P], mst=mst[:M], mst_pat=mp[:M], dist=dist[:len(ids)])

    def route_batches(self, pin_ofs, pins, batch_ofs, net_ids, nthreads=1):
        pin_ofs = np.ascontiguousarray(pin_ofs, dtype=np.int64)
        pins = np.ascontiguousarray(pins, dtype=np.int32)
        batch_ofs = np.ascontiguousarray(batch_ofs, dtype=np.int64)
        ids = np.ascontiguousarray(net_ids, dtype=np.int32)
        M = int((pin_ofs[ids + 1] - pin_ofs[ids]).sum()) if len(ids) else 0
        mst = np.empty(max(M, 1), dtype=np.int64)
        mp = np.empty(max(M, 1), dtype=np.int32)
        rc = lib().gro_route_batches(self._h, _p(pin_ofs), _p(pins), _p(ids), _p(batch_ofs), len(batch_ofs) - 1,
                                     _p(mst), _p(mp), nthreads)
        return rc, mst[:M], mp[:M]

    def count_oob_pairs(self, pin_ofs, pins, net_ids):
        """(pairs, pattern evaluations) for which the reference's L-pattern
        kernel reads a second-via layer v2 == Z past the grid (odd Z)."""
        pin_ofs = np.ascontiguousarray(pin_ofs, dtype=np.int64)
        pins = np.ascontiguousarray(pins, dtype=np.int32)
        ids = np.ascontiguousarray(net_ids, dtype=np.int32)
        out = np.zeros(2, dtype=np.int64)
        lib().gro_count_oob_pairs(self._h, _p(pin_ofs), _p(pins), _p(ids), len(ids), _p(out))
        return int(out[0]), int(out[1])


def batch_pairs(pin_ofs, pins, net_ids) -> np.ndarray:
    pin_ofs = np.ascontiguousarray(pin_ofs, dtype=np.int64)
    pins = np.ascontiguousarray(pins, dtype=np.int32)
    ids = np.ascontiguousarray(net_ids, dtype=np.int32)
    n = int(lib().gro_batch_pairs(_p(pin_ofs), _p(pins), _p(ids), len(ids), None))
    out = np.empty(max(2 * n, 2), dtype=np.int32)
    lib().gro_batch_pairs(_p(pin_ofs), _p(pins), _p(ids), len(ids), _p(out))
    return out[: 2 * n]


def brvsk_net(w, local_id=0):
    w = np.ascontiguousarray(w, dtype=np.float32)
    P = w.size
    n = int(round((1 + (1 + 8 * P) ** 0.5) / 2))
    assert n * (n - 1) // 2 == P
    slots = np.empty(n, dtype=np.int64)
    d = np.empty(1, dtype=np.float32)
    rounds = lib().gro_brvsk_net(n, _p(w), local_id, _p(slots), _p(d))
    return slots, float(d[0]), rounds


def brvsk_build(pin_ofs, net_ids, pair_cost, nthreads=1):
    pin_ofs = np.ascontiguousarray(pin_ofs, dtype=np.int64)
    ids = np.ascontiguousarray(net_ids, dtype=np.int32)
    pc = np.ascontiguousarray(pair_cost, dtype=np.float32)
    M = int((pin_ofs[ids + 1] - pin_ofs[ids]).sum())
    mst = np.empty(max(M, 1), dtype=np.int64)
    dist = np.empty(max(len(ids), 1), dtype=np.float32)
    rc = lib().gro_brvsk_build(_p(pin_ofs), _p(ids), len(ids), _p(pc), _p(mst), _p(dist), nthreads)
    return rc, mst[:M], dist[: len(ids)]
