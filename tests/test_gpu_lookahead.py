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
