"""gr_brvsk_build_static, the Boruvka stage that keeps its scratch in a fixed
device array and allocates nothing: two calls in a row on one stream each
equal gr_brvsk_build on the same batch, bit for bit (edges and FP32 cost
sums -- the tolerance for this index work is zero). The file name puts it
last in collection so it also runs after every other test has used the
device."""
import ctypes as C

import numpy as np
import pytest

import iitmglobalrouter_b200 as gr
from iitmglobalrouter_b200 import _capi


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _design(rng, X, Y, sizes):
    nets = [np.sort(rng.choice(X * Y * 2, size=n, replace=False)).astype(np.int32) for n in sizes]
    ofs = np.cumsum([0] + list(sizes)).astype(np.int64)
    return ofs, np.concatenate(nets)


# net sizes: every k_mst_large shape -- 128 and 512 threads, the matrix in
# shared memory (up to 220 pins) and in the array (221 .. the 1024-pin
# limit), so both of the entry point's launches run; then a batch whose
# largest net fits in shared memory (the first launch only)
MIXES = {
    "to_1024_pins": [2] * 40 + [3, 4, 5, 7, 16, 31, 32, 33, 64, 100, 128, 129, 200, 220, 221, 257, 400, 700, 1024],
    "to_220_pins": [2] * 40 + [3, 4, 5, 7, 16, 31, 32, 33, 64, 100, 128, 129, 200, 220],
}


@pytest.mark.gpu
@pytest.mark.parametrize("mix", sorted(MIXES))
@pytest.mark.parametrize("with_outputs", [True, False], ids=["status_and_dist", "no_status_no_dist"])
def test_static_brvsk_matches_context_entry_point(cuda, mix, with_outputs):
    """Without d_status and d_net_dist the call keeps its status in the
    array and skips the cost sums; the trees are the same."""
    import torch

    X, Y, Z = 64, 64, 4
    rng = np.random.default_rng(7)
    sizes = list(MIXES[mix]) + [int(k) for k in rng.integers(2, 12, size=200)]
    ofs, pins = _design(rng, X, Y, sizes)
    cap = np.ones(X * Y * Z, np.int32)
    R = gr.Router(X, Y, Z, cap)
    R.set_nets(ofs, pins)
    ids = rng.permutation(len(sizes)).astype(np.int32)
    npin = np.ascontiguousarray(np.diff(ofs)[ids], dtype=np.int32)
    P, M = gr.pair_count(ofs, ids), gr.slot_count(ofs, ids)
    L = gr.lib()
    for vals in (4, 1000):  # heavy ties, then few ties; the second call reuses the array
        w = rng.integers(0, vals, size=P).astype(np.float32) * np.float32(0.125)
        w[rng.integers(0, P, size=5)] = np.inf
        dw = torch.from_numpy(w).cuda()
        mst_a = torch.empty(M, dtype=torch.int64, device="cuda")
        dist_a = torch.empty(len(ids), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        R.brvsk_build(ids, dw, mst_a, dist_a)
        R.sync()
        mst_b = torch.full((M,), -7, dtype=torch.int64, device="cuda")
        dist_b = torch.full((len(ids),), float("nan"), dtype=torch.float32, device="cuda")
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream()
        rc = L.gr_brvsk_build_static(npin.ctypes.data_as(C.c_void_p), len(ids), dw.data_ptr(), mst_b.data_ptr(),
                                     dist_b.data_ptr() if with_outputs else None,
                                     status.data_ptr() if with_outputs else None, C.c_void_p(stream.cuda_stream))
        assert rc == 0, _capi.ERRORS.get(rc, rc)
        stream.synchronize()
        assert int(status.item()) == 0
        assert np.array_equal(mst_b.cpu().numpy(), mst_a.cpu().numpy())
        if with_outputs:
            assert np.array_equal(bits(dist_b.cpu().numpy()), bits(dist_a.cpu().numpy()))
        else:
            assert torch.isnan(dist_b).all()  # untouched


def test_static_brvsk_rejects_sizes_beyond_its_limits():
    """Checked on the host before any device work (runs without a GPU)."""
    L = gr.lib()
    one = np.array([_capi.GR_STATIC_MAX_PINS + 1], dtype=np.int32)
    dummy = C.c_void_p(16)  # never dereferenced: the call stops at the size check
    rc = L.gr_brvsk_build_static(one.ctypes.data_as(C.c_void_p), 1, dummy, dummy, None, None, None)
    assert rc == -5  # GR_ERR_NET_TOO_LARGE
    rc = L.gr_brvsk_build_static(one.ctypes.data_as(C.c_void_p), _capi.GR_STATIC_MAX_NETS + 1, dummy, dummy, None,
                                 None, None)
    assert rc == -1  # GR_ERR_ARG
    neg = np.array([-1], dtype=np.int32)
    assert L.gr_brvsk_build_static(neg.ctypes.data_as(C.c_void_p), 1, dummy, dummy, None, None, None) == -1
    assert L.gr_brvsk_build_static(None, 0, None, None, None, None, None) == 0
