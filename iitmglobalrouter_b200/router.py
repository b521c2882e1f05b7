"""Python mirror of the routing hot path's C ABI.

``Router`` wraps a ``gr_ctx`` (grid state on one GPU) and exposes the three
reference boundaries -- ``lpattern`` (BIT_UTIL_SPACE::get_gpu_lpat_dist),
``brvsk_build`` (MST_BUILD::get_mst_tree) and ``mst_bit_commit``
(MST_BIT_COMMIT::bit_commit_edges) -- plus the fused per-batch and per-plan
entry points. Device buffers are torch CUDA tensors; torch only provides
memory and streams, every kernel is the library's own.

``Design`` wraps a ``gr_design`` (host): synthetic generation, the .cap/.net
reader and writer, the -batch_part batcher and the route writer.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import (GR_PLAN_GRAPH, GR_WRT_MERGE, GR_WRT_PPATCH, GR_WRT_RSEG, check, i32, i64, lib, ptr)


class Design:
    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self._lib = lib()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.gr_design_free(h)
            self._h = None

    # ---------------------------------------------------------- construction
    @classmethod
    def generate(cls, config: int, seed: int = 1, n_nets: int = 0) -> "Design":
        h = C.c_void_p()
        check(lib().gr_design_generate(C.byref(h), config, seed, n_nets), "gr_design_generate")
        return cls(h)

    @classmethod
    def generate_custom(cls, X, Y, Z, cap_lo, cap_hi, n_nets, seed=1, hot_frac=0.0, hot_lo=0, hot_hi=0,
                        tail_frac=0.0, tail_hi=61, bbox_median=6.0, bbox_sigma=0.8, pin_layers=2) -> "Design":
        h = C.c_void_p()
        check(lib().gr_design_generate_custom(C.byref(h), X, Y, Z, cap_lo, cap_hi, hot_frac, hot_lo, hot_hi,
                                              n_nets, tail_frac, tail_hi, bbox_median, bbox_sigma, pin_layers,
                                              seed), "gr_design_generate_custom")
        return cls(h)

    @classmethod
    def read(cls, cap_path: str, net_path: str, new_fmt: bool = True) -> "Design":
        h = C.c_void_p()
        check(lib().gr_design_read(C.byref(h), str(cap_path).encode(), str(net_path).encode(), int(new_fmt)),
              "gr_design_read")
        return cls(h)

    def write(self, cap_path: str, net_path: str) -> None:
        check(self._lib.gr_design_write(self._h, str(cap_path).encode(), str(net_path).encode()), "write")

    # ---------------------------------------------------------- contents
    @property
    def dims(self):
        X, Y, Z, n, o = C.c_int(), C.c_int(), C.c_int(), C.c_int32(), C.c_int32()
        p = C.c_int64()
        check(self._lib.gr_design_dims(self._h, C.byref(X), C.byref(Y), C.byref(Z), C.byref(n), C.byref(p),
                                       C.byref(o)))
        return dict(X=X.value, Y=Y.value, Z=Z.value, n_nets=n.value, n_pins=p.value, n_one_pin=o.value)

    def caps(self) -> np.ndarray:
        d = self.dims
        out = np.empty(d["X"] * d["Y"] * d["Z"], dtype=np.int32)
        check(self._lib.gr_design_caps(self._h, ptr(out)), "gr_design_caps")
        return out

    def nets(self):
        d = self.dims
        ofs = np.empty(d["n_nets"] + 1, dtype=np.int64)
        pins = np.empty(max(d["n_pins"], 1), dtype=np.int32)
        check(self._lib.gr_design_nets(self._h, ptr(ofs), ptr(pins)))
        return ofs, pins[: d["n_pins"]]

    def net_name(self, i: int) -> str:
        buf = C.create_string_buffer(4096)
        check(self._lib.gr_design_net_name(self._h, i, buf, 4096))
        return buf.value.decode()

    def batch(self, num_xdim_parts: int = 4):
        """Runs the -batch_part batcher; returns (batch_ofs, net_ids)."""
        nb, ni = C.c_int32(), C.c_int64()
        check(self._lib.gr_design_batch(self._h, num_xdim_parts, C.byref(nb), C.byref(ni)), "gr_design_batch")
        return self.plan()

    def plan(self):
        nb, ni = C.c_int32(), C.c_int64()
        check(self._lib.gr_design_plan(self._h, None, None, C.byref(nb), C.byref(ni)))
        ofs = np.empty(nb.value + 1, dtype=np.int64)
        ids = np.empty(max(ni.value, 1), dtype=np.int32)
        check(self._lib.gr_design_plan(self._h, ptr(ofs), ptr(ids), None, None))
        if nb.value == 0:
            ofs[0] = 0
        return ofs, ids[: ni.value]

    def set_plan(self, batch_ofs, net_ids) -> None:
        batch_ofs, net_ids = i64(batch_ofs), i32(net_ids)
        check(self._lib.gr_design_set_plan(self._h, len(batch_ofs) - 1, ptr(batch_ofs), ptr(net_ids)))

    def write_routes(self, path: str, mst, mst_pat, merge=True, rseg=True, ppatch=True, threads=8):
        mst, mst_pat = i64(mst), i32(mst_pat)
        wv = np.zeros(2, dtype=np.int64)
        flags = (GR_WRT_MERGE if merge else 0) | (GR_WRT_RSEG if rseg else 0) | (GR_WRT_PPATCH if ppatch else 0)
        check(self._lib.gr_design_write_routes(self._h, str(path).encode(), ptr(mst), ptr(mst_pat), flags,
                                               threads, ptr(wv)), "gr_design_write_routes")
        return int(wv[0]), int(wv[1])

    def gather_bytes(self, threads: int = 8) -> dict:
        """Bytes a direct Fenwick evaluation of every pattern of every pin pair
        would gather (4 B per unit: 2 per wire segment, 1 per via cell) and
        the number of valid patterns."""
        out = np.zeros(2, dtype=np.float64)
        check(self._lib.gr_design_gather_bytes(self._h, threads, ptr(out)), "gr_design_gather_bytes")
        return dict(bytes=float(out[0]), patterns=float(out[1]))

    def evaluate(self, demand) -> dict:
        demand = i32(demand)
        out = np.zeros(3, dtype=np.float64)
        check(self._lib.gr_design_eval(self._h, ptr(demand), ptr(out)))
        return dict(overflow=float(out[0]), overflow_cells=int(out[1]), demand=int(out[2]))


def pair_count(pin_ofs: np.ndarray, net_ids: np.ndarray) -> int:
    n = (pin_ofs[net_ids + 1] - pin_ofs[net_ids]).astype(np.int64)
    return int((n * (n - 1) // 2).sum())


def slot_count(pin_ofs: np.ndarray, net_ids: np.ndarray) -> int:
    return int((pin_ofs[net_ids + 1] - pin_ofs[net_ids]).sum())


class Router:
    """A routing context (``gr_ctx``) on one CUDA device."""

    def __init__(self, X: int, Y: int, Z: int, cap, device: int = 0):
        self._lib = lib()
        self.X, self.Y, self.Z = X, Y, Z
        self.csize = X * Y * Z
        cap = i32(cap)
        assert cap.size == self.csize
        h = C.c_void_p()
        check(self._lib.gr_create(C.byref(h), device, X, Y, Z, ptr(cap)), "gr_create")
        self._h = h
        self.device = device
        self._pin_ofs = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gr_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def stream(self) -> int:
        return self._lib.gr_stream(self._h) or 0

    @property
    def launch_count(self) -> int:
        return int(self._lib.gr_launch_count(self._h))

    def reset(self, stream=None):
        check(self._lib.gr_reset(self._h, stream), "gr_reset")

    def set_nets(self, pin_ofs, pins):
        pin_ofs, pins = i64(pin_ofs), i32(pins)
        check(self._lib.gr_set_nets(self._h, len(pin_ofs) - 1, ptr(pin_ofs), ptr(pins)), "gr_set_nets")
        self._pin_ofs = pin_ofs

    # ---------------------------------------------------------- boundaries
    @staticmethod
    def _after_torch(stream, *tensors):
        """With stream None the library works on the context's own stream:
        torch work still queued on the tensors handed over (a fill, a copy)
        finishes first."""
        if stream is not None:
            return
        for t in tensors:
            if t is not None and getattr(t, "is_cuda", False):
                import torch

                torch.cuda.current_stream(t.device).synchronize()
                return

    def lpattern(self, pairs, cost, pat, stream=None):
        """pairs: CUDA int32 [2P]; cost: CUDA float32 [P]; pat: CUDA int16 [P]."""
        n = pairs.numel() // 2
        self._after_torch(stream, pairs, cost, pat)
        check(self._lib.gr_lpattern(self._h, ptr(pairs), n, ptr(cost), ptr(pat), stream), "gr_lpattern")

    def brvsk_build(self, net_ids, pair_cost, mst, dist=None, stream=None):
        ids = i32(net_ids)
        self._after_torch(stream, pair_cost, mst, dist)
        check(self._lib.gr_brvsk_build(self._h, ptr(ids), len(ids), ptr(pair_cost), ptr(mst), ptr(dist), stream),
              "gr_brvsk_build")

    def mst_bit_commit(self, net_ids, mst, pair_pat, mst_pat=None, stream=None):
        ids = i32(net_ids)
        self._after_torch(stream, mst, pair_pat, mst_pat)
        check(self._lib.gr_mst_bit_commit(self._h, ptr(ids), len(ids), ptr(mst), ptr(pair_pat), ptr(mst_pat),
                                          stream), "gr_mst_bit_commit")

    def route_batch(self, net_ids, mst, mst_pat=None, dist=None, pair_cost=None, pair_pat=None, stream=None):
        ids = i32(net_ids)
        self._after_torch(stream, mst, mst_pat, dist, pair_cost, pair_pat)
        check(self._lib.gr_route_batch(self._h, ptr(ids), len(ids), ptr(mst), ptr(mst_pat), ptr(dist),
                                       ptr(pair_cost), ptr(pair_pat), stream), "gr_route_batch")

    # ---------------------------------------------------------- plans
    def plan_set(self, batch_ofs, net_ids):
        batch_ofs, net_ids = i64(batch_ofs), i32(net_ids)
        check(self._lib.gr_plan_set(self._h, len(batch_ofs) - 1, ptr(batch_ofs), ptr(net_ids)), "gr_plan_set")
        self.n_batches = len(batch_ofs) - 1

    @property
    def plan_slots(self) -> int:
        return int(self._lib.gr_plan_slots(self._h))

    def route_plan(self, mst, mst_pat=None, b0=0, b1=None, graph=False, stream=None):
        b1 = self.n_batches if b1 is None else b1
        self._after_torch(stream, mst, mst_pat)
        check(self._lib.gr_route_plan(self._h, b0, b1, ptr(mst), ptr(mst_pat), GR_PLAN_GRAPH if graph else 0,
                                      stream), "gr_route_plan")

    def route_design_host(self, pin_ofs, pins, batch_ofs, net_ids, mst_out, pat_out, graph=False):
        """Upload, plan, route and copy back in one call (host arrays). graph:
        the plan as a CUDA graph, reused while nothing it was built from changes."""
        pin_ofs, pins, batch_ofs, net_ids = i64(pin_ofs), i32(pins), i64(batch_ofs), i32(net_ids)
        check(self._lib.gr_route_design_host(self._h, len(pin_ofs) - 1, ptr(pin_ofs), ptr(pins),
                                             len(batch_ofs) - 1, ptr(batch_ofs), ptr(net_ids), ptr(mst_out),
                                             ptr(pat_out), GR_PLAN_GRAPH if graph else 0), "gr_route_design_host")

    def route_lookahead_host(self, net, every: int, beta: float, mode: str, mst_out, pat_out=None):
        """The uploaded plan routed from reset with the lookahead cost, all in
        the library (gr_route_design_lookahead_host); results into host
        numpy arrays of plan_slots entries."""
        modes = {"demand": _capi.GR_LA_DEMAND, "excess": _capi.GR_LA_EXCESS}
        check(self._lib.gr_route_design_lookahead_host(self._h, net._h, every, C.c_float(beta), modes[mode],
                                                       ptr(mst_out), ptr(pat_out) if pat_out is not None else None),
              "gr_route_design_lookahead_host")

    def route_lookahead_plan(self, net, every: int, beta: float, mode: str, mst, pat=None, graph=True,
                             stream=None):
        """The same learned route into device tensors laid out as route_plan's
        (gr_route_plan_lookahead), as one captured CUDA graph when `graph`;
        enqueued on the context's stream (or `stream`) without waiting."""
        modes = {"demand": _capi.GR_LA_DEMAND, "excess": _capi.GR_LA_EXCESS}
        self._after_torch(stream, mst, pat)
        check(self._lib.gr_route_plan_lookahead(self._h, net._h, every, C.c_float(beta), modes[mode], ptr(mst),
                                                ptr(pat), GR_PLAN_GRAPH if graph else 0, stream),
              "gr_route_plan_lookahead")

    # ---------------------------------------------------------- lookahead
    def features(self, scale: float = 1.0 / 16):
        """Network input from the current state: (2Z, Y, X) CUDA float32."""
        import torch

        out = torch.empty((2 * self.Z, self.Y, self.X), dtype=torch.float32, device=f"cuda:{self.device}")
        torch.cuda.current_stream(self.device).synchronize()  # out allocated and free to write
        check(self._lib.gr_features(self._h, out.data_ptr(), C.c_float(scale), None), "gr_features")
        check(self._lib.gr_sync(self._h), "gr_sync")  # written before other streams read it
        return out

    def set_lookahead(self, pred=None, beta: float = 0.0):
        """pred: (Z, Y, X) CUDA float32 predicted further demand, or None for the plain cost."""
        if pred is not None:
            import torch

            assert pred.is_cuda and pred.dtype == torch.float32 and pred.is_contiguous()
            assert tuple(pred.shape) == (self.Z, self.Y, self.X)
            torch.cuda.current_stream(self.device).synchronize()  # pred complete before this stream reads it
        check(self._lib.gr_set_lookahead(self._h, pred.data_ptr() if pred is not None else None, C.c_float(beta),
                                         None), "gr_set_lookahead")

    # ---------------------------------------------------------- launch shapes
    def tune_set(self, param: int, value: int):
        check(self._lib.gr_tune_set(self._h, param, value), "gr_tune_set")

    def tune_get(self, param: int) -> int:
        v = C.c_int()
        check(self._lib.gr_tune_get(self._h, param, C.byref(v)), "gr_tune_get")
        return v.value

    # ---------------------------------------------------------- profiling
    def profile(self, on: bool = True):
        check(self._lib.gr_profile_enable(self._h, int(on)))

    def profile_read(self, reset: bool = True) -> dict:
        """{kernel name: (milliseconds, launches)} since the last reset."""
        from ._capi import GR_PROF_KINDS
        ms = np.zeros(GR_PROF_KINDS, dtype=np.float64)
        n = np.zeros(GR_PROF_KINDS, dtype=np.int64)
        check(self._lib.gr_profile_read(self._h, ptr(ms), ptr(n), int(reset)), "gr_profile_read")
        return {self._lib.gr_kernel_name(k).decode(): (float(ms[k]), int(n[k])) for k in range(GR_PROF_KINDS)
                if n[k]}

    # ---------------------------------------------------------- state
    def sync(self):
        check(self._lib.gr_sync(self._h), "gr_sync")

    def status(self) -> int:
        return int(self._lib.gr_status(self._h))

    def clear_status(self):
        check(self._lib.gr_clear_status(self._h))

    def capr(self) -> np.ndarray:
        out = np.empty(self.csize, dtype=np.int32)
        check(self._lib.gr_get_capr(self._h, ptr(out)), "gr_get_capr")
        return out

    def demand(self) -> np.ndarray:
        out = np.empty(self.csize, dtype=np.int32)
        check(self._lib.gr_get_demand(self._h, ptr(out)), "gr_get_demand")
        return out

    def fenwick(self) -> np.ndarray:
        out = np.empty(self.csize, dtype=np.float32)
        check(self._lib.gr_get_fenwick(self._h, ptr(out)), "gr_get_fenwick")
        return out
