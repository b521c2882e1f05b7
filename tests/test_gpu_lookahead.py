"""Lookahead routing on the GPU: the network input layout, exact return to
the plain cost, the consistency of the Fenwick trees under the lookahead
cost, and the snapshot -> training -> lookahead-route pipeline."""
import numpy as np
import pytest

import iitmglobalrouter_b200 as gr
import oracle
from iitmglobalrouter_b200 import lookahead

pytestmark = pytest.mark.gpu


def _enc(X, Y, z, x, y):
    return z * X * Y + np.where(z & 1, x * Y + y, y * X + x)


def _setup(config=1, seed=1, n_nets=0):
    import torch

    d = gr.Design.generate(config, seed=seed, n_nets=n_nets)
    dims = d.dims
    bofs, ids = d.batch(4)
    ofs, pins = d.nets()
    R = gr.Router(dims["X"], dims["Y"], dims["Z"], d.caps())
    R.set_nets(ofs, pins)
    R.plan_set(bofs, ids)
    mst = torch.empty(R.plan_slots, dtype=torch.int64, device="cuda")
    pat = torch.empty(R.plan_slots, dtype=torch.int32, device="cuda")
    return d, R, mst, pat, ofs, pins, bofs, ids


def test_features_layout(cuda):
    d, R, mst, pat, *_ = _setup()
    R.route_plan(mst, pat)
    R.sync()
    f = R.features(scale=1.0).cpu().numpy()
    X, Y, Z = R.X, R.Y, R.Z
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    e = _enc(X, Y, z, x, y)
    assert np.array_equal(f[:Z], R.demand()[e].astype(np.float32))
    assert np.array_equal(f[Z:], d.caps()[e].astype(np.float32))


def test_plain_cost_restored_exactly(cuda):
    import torch

    d, R, mst, pat, ofs, pins, bofs, ids = _setup()
    rng = np.random.default_rng(0)
    pred = torch.from_numpy(rng.uniform(0, 3, (R.Z, R.Y, R.X)).astype(np.float32)).cuda()
    R.set_lookahead(pred, 1.0)
    R.reset()
    R.route_plan(mst, pat, b0=0, b1=(len(bofs) - 1) // 2)
    R.sync()
    R.set_lookahead(None)
    R.reset()
    R.route_plan(mst, pat)
    R.sync()
    g = oracle.Grid(R.X, R.Y, R.Z, d.caps())
    rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=8)
    assert rc == 0
    assert np.array_equal(mst.cpu().numpy(), mst_c) and np.array_equal(pat.cpu().numpy(), mp_c)
    assert np.array_equal(R.demand(), g.demand())
    assert np.array_equal(R.fenwick().view(np.uint32), g.fenwick().view(np.uint32))


def test_lookahead_fenwick_matches_rebuild(cuda):
    """Routing with the lookahead cost keeps every Fenwick node equal (to FP32
    rounding) to the node rebuilt from the final capacities."""
    import torch

    d, R, mst, pat, *_ = _setup()
    rng = np.random.default_rng(1)
    pred = torch.from_numpy(rng.uniform(0, 4, (R.Z, R.Y, R.X)).astype(np.float32)).cuda()
    R.set_lookahead(pred, 0.7)
    R.reset()
    R.route_plan(mst, pat)
    R.sync()
    assert R.status() == 0
    inc = R.fenwick()
    R.set_lookahead(pred, 0.7)  # rebuilds from the current capacities
    R.sync()
    reb = R.fenwick()
    np.testing.assert_allclose(inc, reb, rtol=2e-5, atol=1e-6)
    assert int(R.demand().sum()) > 0


def test_snapshot_train_and_route(cuda):
    import torch

    d = gr.Design.generate(1, seed=3)
    samples = lookahead.snapshot_samples(d)
    assert len(samples) == 4
    Z = d.dims["Z"]
    for x, t in samples:
        assert tuple(x.shape) == (2 * Z, d.dims["Y"], d.dims["X"]) and tuple(t.shape) == (Z, d.dims["Y"], d.dims["X"])
        assert float(t.min()) >= 0.0  # demand only grows
    net = lookahead.LookaheadNet(2 * Z, Z, d.dims["Y"], d.dims["X"], hidden=8, n_layers=3, seed=2)
    hist = lookahead.train(net, samples, epochs=30, lr=3e-3)
    assert hist[-1] < hist[0]
    res = lookahead.evaluate(d, net, betas=(0.0, 1.0), every=8)
    plain, la = res[0.0], res[1.0]
    assert plain["demand"] > 0 and la["demand"] > 0 and la["wirelength"] > 0
    # the plain entry is the exact plain route
    _, R, mst, pat, *_ = _setup(1, seed=3)
    R.route_plan(mst, pat)
    R.sync()
    assert plain == lookahead.quality(d, R, mst, pat)


def test_trained_network_lowers_overflow(cuda):
    """The shipped network (trained on snapshots of 50 seeded 400x400x9
    designs) on a design it never saw: lower total overflow than the plain
    cost at no more than 1 % more wirelength."""
    from pathlib import Path

    params = np.load(Path(lookahead.__file__).with_name("lookahead_z9.npy"))
    d = gr.Design.generate(2, seed=1004)
    dims = d.dims
    net = lookahead.LookaheadNet(2 * dims["Z"], dims["Z"], dims["Y"], dims["X"], hidden=32, n_layers=4)
    net.set_params(params)
    res = lookahead.evaluate(d, net, betas=(0.0, 0.5), every=16)
    plain, la = res[0.0], res[0.5]
    assert la["overflow"] < plain["overflow"]
    assert la["wirelength"] <= 1.01 * plain["wirelength"]


def _strong_net(R, Z, seed=5):
    """A random network scaled until its predicted excess over the remaining
    capacity is positive on a few per cent of the cells of the empty grid
    (so both modes change the route)."""
    import torch

    net = lookahead.LookaheadNet(2 * Z, Z, R.Y, R.X, hidden=8, n_layers=3, seed=seed)
    p = net.get_params()
    R.reset()
    f = R.features(lookahead.SCALE)
    for _ in range(12):
        pred = net.forward(f) * (1.0 / lookahead.SCALE)
        if float((torch.relu(pred - (f[Z:] - f[:Z]) * (1.0 / lookahead.SCALE)) > 0).float().mean()) > 0.03:
            break
        p = p * 2.0
        net.set_params(p)
    return net


@pytest.mark.parametrize("mode,beta,every", [("demand", 1.0, 3), ("excess", 0.5, 2), ("excess", 0.0, 4)])
def test_lookahead_host_entry_matches_python_driver(cuda, mode, beta, every):
    """gr_route_design_lookahead_host (network, prediction transform, cost
    switch and routing all inside the library) gives exactly the trees,
    patterns, demand and Fenwick trees of the Python driver; beta 0 is the
    plain route of the oracle."""
    d, R, mst, pat, ofs, pins, bofs, ids = _setup(1, seed=3)
    nb = len(bofs) - 1
    net = _strong_net(R, R.Z)
    lookahead.route_lookahead(R, net, mst, pat, nb, every=every, beta=beta, mode=mode)
    want = (mst.cpu().numpy(), pat.cpu().numpy(), R.demand(), R.fenwick().view(np.uint32))
    R.reset()
    R.route_plan(mst, pat)
    R.sync()
    plain = (mst.cpu().numpy(), pat.cpu().numpy())
    mst_h = np.full(R.plan_slots, -3, np.int64)
    pat_h = np.full(R.plan_slots, -3, np.int32)
    R.route_lookahead_host(net, every, beta, mode, mst_h, pat_h)
    assert np.array_equal(mst_h, want[0]) and np.array_equal(pat_h, want[1])
    assert np.array_equal(R.demand(), want[2])
    assert np.array_equal(R.fenwick().view(np.uint32), want[3])
    if beta > 0:
        assert not (np.array_equal(mst_h, plain[0]) and np.array_equal(pat_h, plain[1]))  # the lookahead acted
    else:
        g = oracle.Grid(R.X, R.Y, R.Z, d.caps())
        rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=8)
        assert rc == 0 and np.array_equal(mst_h, mst_c) and np.array_equal(pat_h, mp_c)


def test_lookahead_host_entry_rejects_mismatched_network(cuda):
    import ctypes as C

    from iitmglobalrouter_b200 import _capi

    d, R, *_ = _setup(1, seed=3)
    net = lookahead.LookaheadNet(2 * R.Z, R.Z, R.Y, R.X + 1, hidden=8, n_layers=2)
    out = np.zeros(R.plan_slots, np.int64)
    L = gr.lib()
    rc = L.gr_route_design_lookahead_host(R._h, net._h, 4, C.c_float(1.0), 0, out.ctypes.data_as(C.c_void_p), None)
    assert rc == -1, _capi.ERRORS.get(rc, rc)
    net = lookahead.LookaheadNet(2 * R.Z, R.Z, R.Y, R.X, hidden=8, n_layers=2)
    for every, beta, mode in ((0, 1.0, 0), (4, -1.0, 0), (4, 1.0, 2)):
        rc = L.gr_route_design_lookahead_host(R._h, net._h, every, C.c_float(beta), mode,
                                              out.ctypes.data_as(C.c_void_p), None)
        assert rc == -1


@pytest.mark.parametrize("mode", ["demand", "excess"])
def test_route_cli_lookahead_matches_python_driver(cuda, tmp_path, mode):
    """`route -lookahead F.npy` (settings from F.json) writes the route file
    that the Python driver's trees and patterns give."""
    import json
    import subprocess

    import torch

    d = gr.Design.generate(1, seed=4)
    cap, net_f, out = tmp_path / "d.cap", tmp_path / "d.net", tmp_path / "d.route"
    d.write(cap, net_f)
    rd = gr.Design.read(cap, net_f)
    dims = rd.dims
    ofs, pins = rd.nets()
    bofs, ids = rd.batch(4)
    R = gr.Router(dims["X"], dims["Y"], dims["Z"], rd.caps())
    R.set_nets(ofs, pins)
    R.plan_set(bofs, ids)
    net = _strong_net(R, R.Z, seed=9)
    np.save(tmp_path / "w.npy", net.get_params().astype(np.float32))
    beta, every = (0.75, 2) if mode == "demand" else (0.5, 3)
    (tmp_path / "w.json").write_text(json.dumps({"hidden": 8, "layers": 3, "every": every, "beta": beta,
                                                 "mode": mode}))
    mst = torch.empty(R.plan_slots, dtype=torch.int64, device="cuda")
    pat = torch.empty(R.plan_slots, dtype=torch.int32, device="cuda")
    lookahead.route_lookahead(R, net, mst, pat, len(bofs) - 1, every=every, beta=beta, mode=mode)
    ref = tmp_path / "py.route"
    rd.write_routes(ref, mst.cpu().numpy(), pat.cpu().numpy(), merge=True, rseg=False, ppatch=False)
    cmd = [str(gr.LIB_PATH.parent / "route"), "-cap", str(cap), "-net", str(net_f), "-gr_out", str(out), "-new_fmt",
           "-bit_pmodel", "-batch_part", "-num_xdim_parts", "4", "-wrt_mrg", "-lookahead", str(tmp_path / "w.npy")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert f"lookahead {mode}" in r.stdout
    assert out.read_bytes() == ref.read_bytes()


def test_lookahead_plan_graph_replays_and_restores_plain_cost(cuda):
    """gr_route_plan_lookahead as one captured graph (network forward passes,
    prediction transforms, Fenwick rebuilds and every batch), captured once
    and replayed: each run equals the stream-ordered run without a graph, and
    afterwards the plain cost is back (a plain route gives the oracle's
    result)."""
    import torch

    d, R, mst, pat, ofs, pins, bofs, ids = _setup(1, seed=3)
    net = _strong_net(R, R.Z)
    R.route_lookahead_plan(net, 4, 1.0, "excess", mst, pat, graph=False)
    R.sync()
    want = (mst.cpu().numpy(), pat.cpu().numpy(), R.demand())
    for _ in range(2):
        mst.fill_(-5)
        torch.cuda.synchronize()
        R.route_lookahead_plan(net, 4, 1.0, "excess", mst, pat, graph=True)
        R.sync()
        assert np.array_equal(mst.cpu().numpy(), want[0]) and np.array_equal(pat.cpu().numpy(), want[1])
        assert np.array_equal(R.demand(), want[2])
        R.reset()
        R.route_plan(mst, pat, graph=True)
        R.sync()
        g = oracle.Grid(R.X, R.Y, R.Z, d.caps())
        rc, mst_c, mp_c = g.route_batches(ofs, pins, bofs, ids, nthreads=8)
        assert rc == 0 and np.array_equal(mst.cpu().numpy(), mst_c) and np.array_equal(pat.cpu().numpy(), mp_c)
    assert R.status() == 0


def test_sharded_samples_through_the_cli_train_like_one_process(cuda, tmp_path, monkeypatch):
    """The training CLI's shard path on the GPU: two ranks' shards (made in
    turn here, RANK / WORLD_SIZE set as torchrun would) hold exactly the
    samples of one process making every seed, and training from them runs."""
    import torch

    for r in range(2):
        monkeypatch.setenv("RANK", str(r))
        monkeypatch.setenv("WORLD_SIZE", "2")
        monkeypatch.setenv("LOCAL_RANK", "0")
        lookahead.main(["--config", "1", "--designs", "3", "--nets", "400", "--shard-dir", str(tmp_path / "s")])
    got = lookahead.load_shards(tmp_path / "s", device="cuda")
    ref = [p for s in range(1, 4) for p in lookahead.snapshot_samples(gr.Design.generate(1, seed=s, n_nets=400))]
    assert len(got) == len(ref) == 12
    for (x, t), (xr, tr) in zip(got, ref):
        assert torch.equal(x, xr) and torch.equal(t, tr)
    rep = lookahead.main(["--config", "1", "--nets", "400", "--samples-dir", str(tmp_path / "s"), "--epochs", "2",
                          "--hidden", "8", "--layers", "2", "--betas", "0,1", "--test-seeds", "9", "--every", "8"])
    assert rep["samples"] == 12 and len(rep["loss"]) == 2
