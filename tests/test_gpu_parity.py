"""GPU parity: the CUDA path against the CPU oracle, bit for bit.

Integer outputs (patterns, MST slots, demand) must be equal; FP32 outputs
(pair costs, Fenwick nodes) must have identical bit patterns -- both sides
perform the same IEEE additions in the same order. All calls go through the
C ABI (ctypes)."""
import numpy as np
import pytest

import iitmglobalrouter_b200 as gr
import oracle

pytestmark = pytest.mark.gpu

NT = 8  # oracle threads


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def dev(torch, a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def design_arrays(d):
    dims = d.dims
    ofs, pins = d.nets()
    return dims["X"], dims["Y"], dims["Z"], d.caps(), ofs, pins


def random_design(X, Y, Z, n_nets, seed, nmax=12, box=6, cap_hi=10):
    rng = np.random.default_rng(seed)
    cap = rng.integers(0, cap_hi + 1, size=X * Y * Z).astype(np.int32)
    g = oracle.Grid(X, Y, Z, cap)
    nets = []
    while len(nets) < n_nets:
        n = int(rng.integers(2, nmax + 1))
        w, h = int(rng.integers(1, box + 1)), int(rng.integers(1, box + 1))
        x0, y0 = int(rng.integers(0, X - w + 1)), int(rng.integers(0, Y - h + 1))
        pins = sorted({g.enc(int(rng.integers(0, min(Z, 3))), x0 + int(rng.integers(0, w)), y0 + int(rng.integers(0, h)))
                       for _ in range(n)})
        if len(pins) >= 2:
            nets.append(pins)
    ofs = np.cumsum([0] + [len(q) for q in nets]).astype(np.int64)
    pins = np.concatenate([np.array(q, np.int32) for q in nets])
    return cap, ofs, pins


def simple_batches(n, size):
    ids = np.arange(n, dtype=np.int32)
    bofs = np.arange(0, n + size, size)
    bofs[-1] = n
    return np.unique(bofs).astype(np.int64), ids


@pytest.mark.parametrize("Z", [3, 5, 9, 10])
def test_lpattern_boundary_bitexact(cuda, Z):
    import torch

    X, Y = 23, 17
    cap, ofs, pins = random_design(X, Y, Z, 60, Z)
    g = oracle.Grid(X, Y, Z, cap)
    R = gr.Router(X, Y, Z, cap)
    R.set_nets(ofs, pins)
    # move the cost state away from its initial values: route some batches
    bofs, ids = simple_batches(60, 15)
    for b in range(len(bofs) - 1):
        sl = ids[bofs[b]:bofs[b + 1]]
        g.route_batch(ofs, pins, sl, nthreads=NT)
        M = gr.slot_count(ofs, sl)
        mst = torch.empty(M, dtype=torch.int64, device="cuda")
        R.route_batch(sl, mst)
    R.sync()
    assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))
    rng = np.random.default_rng(7)
    pairs = rng.integers(0, X * Y * Z, size=(4000, 2)).astype(np.int32)
    e = rng.integers(0, X * Y * Z, size=300)
    zz, r = e // (X * Y), e % (X * Y)
    stacked = np.stack([e, ((zz + 1) % Z) * X * Y + r], 1)  # same (x,y) on another layer
    pairs = np.vstack([pairs, stacked, pairs[:10, ::-1]]).astype(np.int32)
    ccpu, pcpu = g.lpattern(pairs.ravel(), nthreads=NT)
    dp = dev(torch, pairs.ravel())
    cost = torch.empty(len(pairs), dtype=torch.float32, device="cuda")
    pat = torch.empty(len(pairs), dtype=torch.int16, device="cuda")
    torch.cuda.synchronize()
    R.lpattern(dp, cost, pat)
    R.sync()
    assert np.array_equal(pat.cpu().numpy(), pcpu)
    assert np.array_equal(bits(cost.cpu().numpy()), bits(ccpu))
    assert R.status() == 0


def test_brvsk_boundary_bitexact(cuda):
    import torch

    X, Y, Z = 40, 40, 4
    rng = np.random.default_rng(3)
    sizes = [2, 3, 4, 5, 7, 16, 33, 64, 100, 257]
    g = oracle.Grid(X, Y, Z, np.ones(X * Y * Z, np.int32))
    nets = []
    for n in sizes:
        cells = rng.choice(X * Y * 2, size=n, replace=False)
        nets.append(np.sort(cells).astype(np.int32))
    ofs = np.cumsum([0] + [len(q) for q in nets]).astype(np.int64)
    pins = np.concatenate(nets)
    R = gr.Router(X, Y, Z, np.ones(X * Y * Z, np.int32))
    R.set_nets(ofs, pins)
    ids = rng.permutation(len(nets)).astype(np.int32)
    P = gr.pair_count(ofs, ids)
    M = gr.slot_count(ofs, ids)
    for trial, vals in enumerate([4, 1000]):  # heavy ties, then few ties
        w = (rng.integers(0, vals, size=P).astype(np.float32) * np.float32(0.125))
        w[rng.integers(0, P, size=5)] = np.inf
        rc, mst_c, dist_c = oracle.brvsk_build(ofs, ids, w, nthreads=NT)
        assert rc == 0
        mst = torch.empty(M, dtype=torch.int64, device="cuda")
        dist = torch.empty(len(ids), dtype=torch.float32, device="cuda")
        dw = dev(torch, w)
        torch.cuda.synchronize()
        R.brvsk_build(ids, dw, mst, dist)
        R.sync()
        assert np.array_equal(mst.cpu().numpy(), mst_c)
        assert np.array_equal(bits(dist.cpu().numpy()), bits(dist_c))


# (mid threads, big threads, cluster threads, cluster from pins[, L-pattern split, persistent queue])
TUNINGS = [(128, 256, 256, 0), (1024, 1024, 1024, 129), (256, 512, 512, 200), (64, 64, 64, 0),
           (1024, 1024, 1024, 129, 0, 1)]


@pytest.mark.parametrize("tuning", TUNINGS)
def test_brvsk_launch_shapes_do_not_change_results(cuda, tuning):
    """Every Boruvka launch shape gives the oracle's trees bit for bit: nets
    in the mid class, single-CTA big nets, 4- and 8-CTA clusters and the
    global-matrix path (700 pins); and the persistent queue kernel, which
    takes all of them (the 700-pin net through its global matrix)."""
    import torch

    X, Y, Z = 48, 48, 4
    rng = np.random.default_rng(11)
    sizes = [2, 3, 33, 64, 128, 129, 150, 200, 220, 221, 300, 450, 700] + [int(k) for k in rng.integers(2, 40, 30)]
    nets = [np.sort(rng.choice(X * Y * 2, size=n, replace=False)).astype(np.int32) for n in sizes]
    ofs = np.cumsum([0] + sizes).astype(np.int64)
    pins = np.concatenate(nets)
    R = gr.Router(X, Y, Z, np.ones(X * Y * Z, np.int32))
    R.set_nets(ofs, pins)
    for p, v in enumerate(tuning):
        R.tune_set(p, v)
        assert R.tune_get(p) == v
    ids = rng.permutation(len(sizes)).astype(np.int32)
    P, M = gr.pair_count(ofs, ids), gr.slot_count(ofs, ids)
    w = rng.integers(0, 50, size=P).astype(np.float32) * np.float32(0.25)
    rc, mst_c, dist_c = oracle.brvsk_build(ofs, ids, w, nthreads=NT)
    assert rc == 0
    mst = torch.empty(M, dtype=torch.int64, device="cuda")
    dist = torch.empty(len(ids), dtype=torch.float32, device="cuda")
    R.brvsk_build(ids, dev(torch, w), mst, dist)
    R.sync()
    assert np.array_equal(mst.cpu().numpy(), mst_c)
    assert np.array_equal(bits(dist.cpu().numpy()), bits(dist_c))


def test_tune_rejects_bad_values(cuda):
    R = gr.Router(8, 8, 3, np.ones(192, np.int32))
    for p, v in [(0, 48), (0, 2048), (1, 100), (3, 100), (3, 5000), (4, 3), (4, 8), (5, 2), (5, -1), (7, 512)]:
        with pytest.raises(gr.GRError):
            R.tune_set(p, v)


def test_commit_boundary_bitexact(cuda):
    import torch

    X, Y, Z = 31, 29, 6
    cap, ofs, pins = random_design(X, Y, Z, 80, 11, nmax=9)
    g = oracle.Grid(X, Y, Z, cap)
    R = gr.Router(X, Y, Z, cap)
    R.set_nets(ofs, pins)
    ids = np.arange(0, 80, 2, dtype=np.int32)  # arbitrary nets: boxes may overlap
    r = g.route_batch(ofs, pins, ids, nthreads=NT)  # oracle lpattern + brvsk + commit
    mst = dev(torch, r["mst"])
    pp = dev(torch, r["pair_pat"])
    mp = torch.empty(len(r["mst"]), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    R.mst_bit_commit(ids, mst, pp, mp)
    R.sync()
    assert np.array_equal(mp.cpu().numpy(), r["mst_pat"])
    assert np.array_equal(R.capr(), g.capr())
    assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))


def route_all_gpu(R, ofs, bofs, ids, mode):
    import torch

    M = gr.slot_count(ofs, ids)
    mst = torch.full((M,), -7, dtype=torch.int64, device="cuda")
    mp = torch.full((M,), -7, dtype=torch.int32, device="cuda")
    if mode == "batch":
        slot = 0
        for b in range(len(bofs) - 1):
            sl = ids[bofs[b]:bofs[b + 1]]
            m = gr.slot_count(ofs, sl)
            R.route_batch(sl, mst[slot:slot + m], mp[slot:slot + m])
            slot += m
    else:
        R.plan_set(bofs, ids)
        R.route_plan(mst, mp, graph=(mode == "graph"))
    R.sync()
    return mst.cpu().numpy(), mp.cpu().numpy()


@pytest.mark.parametrize("mode", ["batch", "plan", "graph"])
def test_route_config1_bitexact(cuda, mode):
    """The 64x64x5 design (2,000 nets), -batch_part -num_xdim_parts 4, all
    batches: MST slots, patterns, demand and every Fenwick node."""
    d = gr.Design.generate(1, seed=1)
    X, Y, Z, cap, ofs, pins = design_arrays(d)
    bofs, ids = d.batch(4)
    g = oracle.Grid(X, Y, Z, cap)
    rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
    assert rc == 0
    R = gr.Router(X, Y, Z, cap)
    R.set_nets(ofs, pins)
    mst, mp = route_all_gpu(R, ofs, bofs, ids, mode)
    assert np.array_equal(mst, mst_c)
    assert np.array_equal(mp, mp_c)
    assert np.array_equal(R.demand(), g.demand())
    assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))
    assert R.status() == 0


@pytest.mark.parametrize("mode", ["plan", "graph"])
def test_route_persistent_queue_bitexact(cuda, mode):
    """The whole 64x64x5 route and the first batches of the 400x400x9 design
    with every batch's Boruvka stage in one persistent queue launch: the
    oracle's trees, patterns, capacities and Fenwick nodes."""
    from iitmglobalrouter_b200._capi import GR_TUNE_MST_QUEUE

    for config, n_nets, nb in ((1, 0, None), (2, 40000, 3)):
        d = gr.Design.generate(config, seed=2, n_nets=n_nets)
        X, Y, Z, cap, ofs, pins = design_arrays(d)
        bofs, ids = d.batch(4)
        if nb is not None:
            bofs, ids = bofs[: nb + 1], ids[: bofs[nb]]
        g = oracle.Grid(X, Y, Z, cap)
        rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
        assert rc == 0
        R = gr.Router(X, Y, Z, cap)
        R.set_nets(ofs, pins)
        R.tune_set(GR_TUNE_MST_QUEUE, 1)
        for _ in range(2):  # the queue counters are back at zero for the second route
            R.reset()
            mst, mp = route_all_gpu(R, ofs, bofs, ids, mode)
            assert np.array_equal(mst, mst_c)
            assert np.array_equal(mp, mp_c)
            assert np.array_equal(R.capr(), g.capr())
            assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))
            assert R.status() == 0


@pytest.mark.parametrize("X,Y,Z", [(37, 53, 5), (64, 64, 4), (3100, 6, 3)])
def test_fenwick_build_bitexact(cuda, X, Y, Z):
    """The Fenwick trees of a reset (one warp per track, levels built from
    their left halves; the per-cell kernel for tracks above 3072 cells)
    equal the oracle's bit for bit."""
    rng = np.random.default_rng(X * Y + Z)
    cap = rng.integers(-3, 40, size=X * Y * Z).astype(np.int32)
    R = gr.Router(X, Y, Z, cap)
    R.reset()
    g = oracle.Grid(X, Y, Z, cap)
    assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))


def test_plan_descriptor_built_on_device_matches_host_builder(cuda):
    """gr_plan_set builds the plan's descriptor on the device: equal, array by
    array and batch total by batch total, to the host builder's, for the
    generated plans and for a plan with an empty batch and nets of every size
    class (2, 3..32, 33..128, above 128 pins); ids outside the design are
    rejected."""
    L = gr.lib()
    for config, n_nets in ((1, 0), (2, 30000)):
        d = gr.Design.generate(config, seed=5, n_nets=n_nets)
        X, Y, Z, cap, ofs, pins = design_arrays(d)
        bofs, ids = d.batch(4)
        R = gr.Router(X, Y, Z, cap)
        R.set_nets(ofs, pins)
        R.plan_set(bofs, ids)
        assert L.gr_plan_check(R._h) == 0
    X, Y, Z = 40, 40, 4
    rng = np.random.default_rng(3)
    sizes = [2, 3, 32, 33, 128, 129, 300, 2, 5, 17, 2, 64, 200] + [int(k) for k in rng.integers(2, 40, 300)]
    nets = [np.sort(rng.choice(X * Y * 2, size=n, replace=False)).astype(np.int32) for n in sizes]
    ofs = np.cumsum([0] + sizes).astype(np.int64)
    R = gr.Router(X, Y, Z, np.ones(X * Y * Z, np.int32))
    R.set_nets(ofs, np.concatenate(nets))
    ids = rng.permutation(len(sizes)).astype(np.int32)
    bofs = np.array([0, 7, 7, 150, len(sizes)], np.int64)  # the second batch is empty
    R.plan_set(bofs, ids)
    assert L.gr_plan_check(R._h) == 0
    bad = ids.copy()
    bad[100] = len(sizes)
    with pytest.raises(gr.GRError):
        R.plan_set(bofs, bad)


def test_route_config2_first_batches_bitexact(cuda):
    """The 400x400x9 design (odd Z), first batches of the -batch_part plan."""
    d = gr.Design.generate(2, seed=1, n_nets=40000)
    X, Y, Z, cap, ofs, pins = design_arrays(d)
    bofs, ids = d.batch(4)
    nb = 3
    bofs, ids = bofs[: nb + 1], ids[: bofs[nb]]
    g = oracle.Grid(X, Y, Z, cap)
    rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
    assert rc == 0
    R = gr.Router(X, Y, Z, cap)
    R.set_nets(ofs, pins)
    mst, mp = route_all_gpu(R, ofs, bofs, ids, "plan")
    assert np.array_equal(mst, mst_c)
    assert np.array_equal(mp, mp_c)
    assert np.array_equal(R.capr(), g.capr())
    assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))


def test_large_nets_direct_query_path(cuda):
    """Nets above the per-net query-table size use direct Fenwick gathers."""
    X, Y, Z = 64, 64, 4
    rng = np.random.default_rng(5)
    cap = rng.integers(2, 9, size=X * Y * Z).astype(np.int32)
    g = oracle.Grid(X, Y, Z, cap)
    big = np.sort(rng.choice(X * Y * 2, size=1100, replace=False)).astype(np.int32)
    small = np.sort(rng.choice(X * Y * 2, size=40, replace=False)).astype(np.int32)
    ofs = np.array([0, len(big), len(big) + len(small)], np.int64)
    pins = np.concatenate([big, small])
    bofs, ids = np.array([0, 1, 2], np.int64), np.array([0, 1], np.int32)
    rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
    assert rc == 0
    R = gr.Router(X, Y, Z, cap)
    R.set_nets(ofs, pins)
    mst, mp = route_all_gpu(R, ofs, bofs, ids, "plan")
    assert np.array_equal(mst, mst_c) and np.array_equal(mp, mp_c)
    assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))


def test_edge_cases_small_grids(cuda):
    """Z = 3, one-row tracks, all pins on one track, stacked pins."""
    import torch

    for (X, Y, Z) in [(1, 9, 3), (9, 1, 3), (2, 2, 3), (5, 4, 7)]:
        cap = np.arange(X * Y * Z, dtype=np.int32) % 5
        g = oracle.Grid(X, Y, Z, cap)
        cells = [g.enc(z, x, y) for z in range(min(Z, 3)) for x in range(X) for y in range(Y)]
        nets = [sorted(cells[:2]), sorted(cells[-3:]), sorted(cells[:: max(1, len(cells) // 5)])]
        nets = [q for q in nets if len(set(q)) >= 2]
        ofs = np.cumsum([0] + [len(q) for q in nets]).astype(np.int64)
        pins = np.concatenate([np.array(q, np.int32) for q in nets])
        bofs = np.arange(len(nets) + 1, dtype=np.int64)
        ids = np.arange(len(nets), dtype=np.int32)
        rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids)
        assert rc == 0
        R = gr.Router(X, Y, Z, cap)
        R.set_nets(ofs, pins)
        mst, mp = route_all_gpu(R, ofs, bofs, ids, "batch")
        assert np.array_equal(mst, mst_c) and np.array_equal(mp, mp_c), (X, Y, Z)
        assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))
        # an empty batch is a no-op
        R.route_batch(np.array([], np.int32), torch.empty(1, dtype=torch.int64, device="cuda"))
        R.sync()


@pytest.mark.parametrize("X", [300, 1000])
def test_dense_tracks_bitexact(cuda, X):
    """Batches that mark hundreds of cells of one track (rows of disjoint
    2-pin nets along x): the commit updates such tracks node by node. Track
    lengths 300 and 1000 start at cells that are not multiples of 32."""
    Y, Z = 7, 3
    cap = (np.arange(X * Y * Z, dtype=np.int32) % 7 + 3).astype(np.int32)
    g = oracle.Grid(X, Y, Z, cap)
    nets = []
    for shift in (0, 4):  # the second batch overlaps the first one's wires
        for y in range(Y):
            for x0 in range(shift, X - 9, 10):
                nets.append(sorted({g.enc(0, x0, y), g.enc(0, x0 + 8, y), g.enc(y % 2, x0 + 3, y)}))
    ofs = np.cumsum([0] + [len(q) for q in nets]).astype(np.int64)
    pins = np.concatenate([np.array(q, np.int32) for q in nets])
    half = len(nets) // 2
    bofs = np.array([0, half, len(nets)], np.int64)
    ids = np.arange(len(nets), dtype=np.int32)
    rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
    assert rc == 0
    R = gr.Router(X, Y, Z, cap)
    R.set_nets(ofs, pins)
    mst, mp = route_all_gpu(R, ofs, bofs, ids, "plan")
    assert np.array_equal(mst, mst_c) and np.array_equal(mp, mp_c)
    assert np.array_equal(R.capr(), g.capr())
    assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))
    # some track of layer 2 gained more than 64 units of demand in one batch
    dem = (cap - R.capr()).reshape(Z, Y, X)
    assert int((dem[2] > 0).sum(axis=1).max()) > 64


def test_invalid_inputs_reported_not_faulted(cuda):
    import torch

    X, Y, Z = 8, 8, 4
    cap = np.full(X * Y * Z, 5, np.int32)
    R = gr.Router(X, Y, Z, cap)
    g = oracle.Grid(X, Y, Z, cap)
    pins = np.array(sorted([g.enc(0, 1, 2), g.enc(0, 5, 2)]), np.int32)
    R.set_nets(np.array([0, 2]), pins)
    mp = torch.empty(2, dtype=torch.int32, device="cuda")
    # pattern 0 has via1 = 0: not a pattern
    R.mst_bit_commit([0], dev(torch, np.array([1, -1])), dev(torch, np.array([0], np.int16)), mp)
    assert R.status() & gr._capi.GR_ST_BAD_PATTERN
    R.clear_status()
    # slot naming a pin outside the net
    R.mst_bit_commit([0], dev(torch, np.array([(0 << 15) | 5, -1])), dev(torch, np.array([4], np.int16)), mp)
    assert R.status() & gr._capi.GR_ST_BAD_EDGE
    R.clear_status()
    # pair outside the grid
    cost = torch.empty(1, dtype=torch.float32, device="cuda")
    pat = torch.empty(1, dtype=torch.int16, device="cuda")
    R.lpattern(dev(torch, np.array([0, X * Y * Z + 3], np.int32)), cost, pat)
    assert R.status() & gr._capi.GR_ST_BAD_PIN
    R.clear_status()
    with pytest.raises(gr.GRError):
        R.set_nets(np.array([0, 1]), np.array([3], np.int32))  # one-pin net
    with pytest.raises(gr.GRError):
        R.route_batch(np.array([5], np.int32), torch.empty(4, dtype=torch.int64, device="cuda"))  # bad id
    assert R.status() == 0


def test_route_design_host_end_to_end(cuda):
    d = gr.Design.generate(1, seed=2)
    X, Y, Z, cap, ofs, pins = design_arrays(d)
    bofs, ids = d.batch(4)
    g = oracle.Grid(X, Y, Z, cap)
    rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
    R = gr.Router(X, Y, Z, cap)
    M = gr.slot_count(ofs, ids)
    mst, mp = np.empty(M, np.int64), np.empty(M, np.int32)
    R.route_design_host(ofs, pins, bofs, ids, mst, mp)
    assert np.array_equal(mst, mst_c) and np.array_equal(mp, mp_c)
    assert np.array_equal(R.demand(), g.demand())


def test_route_design_host_graph_reuse(cuda):
    """The host-buffer entry in graph mode, called repeatedly on one context:
    a graph is replayed while its plan's shapes and buffers are unchanged and
    rebuilt when the design changes; every call gives the oracle's result,
    with page-locked and with pageable output buffers."""
    import torch

    designs = [gr.Design.generate(1, seed=s) for s in (1, 2)]
    X, Y, Z, cap, _, _ = design_arrays(designs[0])  # the second design's nets on the first one's grid
    ref = []
    for d in designs:
        _, _, _, _, ofs, pins = design_arrays(d)
        bofs, ids = d.batch(4)
        g = oracle.Grid(X, Y, Z, cap)
        rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
        assert rc == 0
        ref.append((ofs, pins, bofs, ids, mst_c, mp_c, g.demand()))
    R = gr.Router(X, Y, Z, cap)
    for k in (0, 0, 1, 0, 1, 1):
        ofs, pins, bofs, ids, mst_c, mp_c, dem = ref[k]
        for pinned in (True, False):
            M = len(mst_c)
            if pinned:
                h_mst = torch.full((M,), -9, dtype=torch.int64).pin_memory().numpy()
                h_pat = torch.full((M,), -9, dtype=torch.int32).pin_memory().numpy()
            else:
                h_mst, h_pat = np.full(M, -9, np.int64), np.full(M, -9, np.int32)
            R.route_design_host(ofs, pins, bofs, ids, h_mst, h_pat, graph=True)
            assert np.array_equal(h_mst, mst_c) and np.array_equal(h_pat, mp_c)
            assert np.array_equal(R.demand(), dem)


def test_contexts_of_different_sizes_coexist(cuda):
    """A context for a small grid created after one for a larger grid leaves
    the larger one routable (kernel attributes are process-wide)."""
    d = gr.Design.generate_custom(300, 300, 3, 2, 6, 400, seed=1)
    X, Y, Z, cap, ofs, pins = design_arrays(d)
    bofs, ids = d.batch(4)
    big = gr.Router(X, Y, Z, cap)
    big.set_nets(ofs, pins)
    a, _ = route_all_gpu(big, ofs, bofs, ids, "plan")
    small = gr.Router(16, 16, 3, np.ones(16 * 16 * 3, np.int32))
    big.reset()
    b, _ = route_all_gpu(big, ofs, bofs, ids, "plan")
    assert big.status() == 0 and np.array_equal(a, b)
    small.close()


@pytest.mark.parametrize("split", [1, 2, 4])
def test_lpattern_split_bitexact(cuda, split):
    """The L-pattern kernel with the first-via layers of each pair shared by
    1, 2 or 4 warps gives the oracle's routes (even and odd Z)."""
    from iitmglobalrouter_b200._capi import GR_TUNE_LPAT_SPLIT

    for config, n_nets, nb in ((1, 0, None), (2, 20000, 2)):
        d = gr.Design.generate(config, seed=2, n_nets=n_nets)
        X, Y, Z, cap, ofs, pins = design_arrays(d)
        bofs, ids = d.batch(4)
        if nb:
            bofs, ids = bofs[: nb + 1], ids[: bofs[nb]]
        g = oracle.Grid(X, Y, Z, cap)
        rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=NT)
        assert rc == 0
        R = gr.Router(X, Y, Z, cap)
        R.tune_set(GR_TUNE_LPAT_SPLIT, split)
        R.set_nets(ofs, pins)
        mst, mp = route_all_gpu(R, ofs, bofs, ids, "plan")
        assert np.array_equal(mst, mst_c) and np.array_equal(mp, mp_c)
        assert np.array_equal(bits(R.fenwick()), bits(g.fenwick()))


def test_traffic_helper_units(cuda, tmp_path):
    """The profile helper's route: the units of the captured batches (pairs
    per class from the plan, committed GCELLs from the demand they add) on a
    small design, with the router's own demand as the check."""
    import json

    from iitmglobalrouter_b200 import traffic

    out = tmp_path / "u.json"
    traffic.route(type("A", (), {"config": 1, "seed": 1, "batches": "2:4", "units": str(out)})())
    u = json.loads(out.read_text())["units"]
    d = gr.Design.generate(1, seed=1)
    ofs, pins = d.nets()
    bofs, ids = d.batch(4)
    pairs = gr.pair_count(ofs, ids[bofs[2]:bofs[4]])
    assert u["k_lpat"] == pairs > 0
    assert u["k_mst_large"] + u["k_mst_warp"] <= pairs and u["k_qtable"] > 0
    assert u["k_track_commit"] > 0
