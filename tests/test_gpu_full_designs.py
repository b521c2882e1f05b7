"""GPU parity on whole designs: every batch of the 400x400x9 design (150 K
nets, odd Z) and of the 1.2M-net 1000x1000x10 design that the benchmark
routes, through the captured-graph plan route, against the CPU oracle.

Bit for bit: every MST slot, every slot's pattern, the remaining capacity of
every GCELL and every Fenwick node (FP32 bit patterns), after the last
batch -- any difference in any batch propagates into the cost state of all
later ones. The 400x400x9 case also counts the pairs for which the
reference's own kernel would evaluate a second-via layer past the top layer
(odd Z, bit_util.hpp:157-164), which the oracle and this library treat as
invalid patterns."""
import os

import numpy as np
import pytest

import iitmglobalrouter_b200 as gr
import oracle

pytestmark = pytest.mark.gpu

NT = os.cpu_count() or 8


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def route_full(config, seed):
    import torch

    d = gr.Design.generate(config, seed=seed)
    dims = d.dims
    X, Y, Z = dims["X"], dims["Y"], dims["Z"]
    cap = d.caps()
    ofs, pins = d.nets()
    bofs, ids = d.batch(4)
    R = gr.Router(X, Y, Z, cap)
    R.set_nets(ofs, pins)
    R.plan_set(bofs, ids)
    M = R.plan_slots
    mst = torch.empty(M, dtype=torch.int64, device="cuda")
    pat = torch.empty(M, dtype=torch.int32, device="cuda")
    R.route_plan(mst, pat, graph=True)
    R.sync()
    gpu = dict(mst=mst.cpu().numpy(), pat=pat.cpu().numpy(), capr=R.capr(), fen=R.fenwick(), status=R.status())
    R.close()
    del mst, pat
    torch.cuda.empty_cache()
    g = oracle.Grid(X, Y, Z, cap)
    rc, mst_c, pat_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
    assert rc == 0
    return d, g, (ofs, pins, bofs, ids), gpu, (mst_c, pat_c)


def check(g, gpu, ref):
    mst_c, pat_c = ref
    assert gpu["status"] == 0
    assert len(gpu["mst"]) == len(mst_c)
    bad = np.flatnonzero(gpu["mst"] != mst_c)
    assert bad.size == 0, f"{bad.size} MST slots differ, first at slot {bad[:5]}"
    bad = np.flatnonzero(gpu["pat"] != pat_c)
    assert bad.size == 0, f"{bad.size} slot patterns differ, first at slot {bad[:5]}"
    assert np.array_equal(gpu["capr"], g.capr())
    assert np.array_equal(bits(gpu["fen"]), bits(g.fenwick()))


def test_route_400x400x9_all_batches_bitexact(cuda):
    """150 K nets (0.5 % tail of 61..200 pins), 232 batches of -batch_part
    -num_xdim_parts 4, Z = 9."""
    d, g, (ofs, pins, bofs, ids), gpu, ref = route_full(2, 1)
    assert len(bofs) - 1 > 200 and np.diff(ofs).max() > 60
    check(g, gpu, ref)
    pairs, evals = g.count_oob_pairs(ofs, pins, ids)
    # every pair whose pins differ in x and y has the four patterns via1 in
    # {2, 4, 6, 8}, v = 4, whose second via would be layer 9
    assert pairs > 0 and evals == 4 * pairs
    print(f"\n400x400x9: {gr.pair_count(ofs, ids)} pairs; the reference reads layer Z=9 out of bounds "
          f"for {pairs} of them ({evals} pattern evaluations)")


@pytest.mark.slow
def test_route_1200k_nets_all_batches_bitexact(cuda):
    """The benchmark's workload: 1,195,755 nets (1 % tail up to 400 pins),
    559 batches, 1000x1000x10."""
    d, g, (ofs, pins, bofs, ids), gpu, ref = route_full(3, 1)
    assert len(ids) > 1_000_000 and np.diff(ofs).max() > 300
    check(g, gpu, ref)
    assert g.count_oob_pairs(ofs, pins, ids[:1000]) == (0, 0)  # even Z: no second via past the grid
