"""The congestion lookahead network: the CUDA GEMM, forward pass and
gradients against the float64 restatement in tests/cnnref.py (which rounds
the GEMM operands to BF16 as the kernels do), and the restatement itself
against finite differences."""
import numpy as np
import pytest

import cnnref


def test_reference_gradients_match_finite_differences(monkeypatch):
    """The restatement's backward pass, with its BF16 and FP32 rounding switched off."""
    exact = lambda x: np.asarray(x, dtype=np.float64)  # noqa: E731
    monkeypatch.setattr(cnnref, "q", exact)
    monkeypatch.setattr(cnnref, "f32", exact)
    rng = np.random.default_rng(0)
    shapes = [(2, 3), (3, 3), (3, 2)]
    n = sum(co * ci * 9 + co for ci, co in shapes)
    p = rng.normal(0, 0.5, n)
    x = rng.normal(0, 1, (2, 5, 4))
    t = rng.normal(0, 1, (2, 5, 4))
    _, g = cnnref.grads(p, shapes, x, t)
    for i in rng.choice(n, 12, replace=False):
        e = np.zeros(n)
        e[i] = 1e-5
        lp = cnnref.grads(p + e, shapes, x, t)[0]
        lm = cnnref.grads(p - e, shapes, x, t)[0]
        assert g[i] == pytest.approx((lp - lm) / 2e-5, rel=1e-5, abs=1e-8)


def _bf16_matrix(rng, shape):
    return cnnref.bf16(rng.normal(0, 1, shape).astype(np.float32)).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,splits", [(100, 20, 40, 1), (64, 32, 16, 1), (257, 9, 288, 4), (33, 40, 170, 3)])
def test_gemm_matches_numpy(cuda, M, N, K, splits):
    import torch

    import iitmglobalrouter_b200 as gr

    rng = np.random.default_rng(M + N + K)
    a, b = _bf16_matrix(rng, (M, K)), _bf16_matrix(rng, (K, N))
    da = torch.from_numpy(a).cuda().to(torch.bfloat16)  # exact: the values are BF16
    db = torch.from_numpy(b).cuda().to(torch.bfloat16)
    dc = torch.empty((M, N), dtype=torch.float32, device="cuda")
    assert gr.lib().gr_cnn_gemm_test(M, N, K, da.data_ptr(), db.data_ptr(), dc.data_ptr(), splits) == 0
    ref = a.astype(np.float64) @ b.astype(np.float64)
    np.testing.assert_allclose(dc.cpu().numpy(), ref, rtol=1e-5, atol=1e-4)


def _net_case(seed=3, H=12, W=10, cin=4, cout=2, hidden=8, layers=3):
    from iitmglobalrouter_b200.lookahead import LookaheadNet

    rng = np.random.default_rng(seed)
    net = LookaheadNet(cin, cout, H, W, hidden=hidden, n_layers=layers, seed=seed)
    x = rng.uniform(0, 1, (cin, H, W)).astype(np.float32)
    t = rng.uniform(0, 1, (cout, H, W)).astype(np.float32)
    return net, x, t


def _bf16_round(a):
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("H,W,cin,hidden,cout", [
    (37, 29, 20, 32, 20),  # one ragged strip of 29 of 128 positions per row; 20 channels padded to 32; 32 output columns
    (16, 8, 32, 16, 10),  # strips of 8 positions; 32 channels; 16 output columns
    (50, 50, 32, 32, 32),  # 50 strips
    (6, 300, 20, 16, 16),  # three strips per row, the last ragged (300 = 2 x 128 + 44)
])
def test_forward_exact_on_binary_grid(cuda, H, W, cin, hidden, cout):
    """Inputs on multiples of 1/16 in [0, 4) and weights on multiples of 1/64
    in [-1, 1]: every first-layer sum is exact in FP32 whatever the order of
    accumulation, and the second layer copies channel j of the (BF16-rounded)
    ReLU output to output j through its centre tap. The forward must then equal
    the float64 value bit for bit -- gather, shared-memory layout, tensor-core
    tiles, bias, ReLU and the ragged last tile all checked exactly."""
    import torch

    from iitmglobalrouter_b200.lookahead import LookaheadNet

    rng = np.random.default_rng(H * W + cin)
    net = LookaheadNet(cin, cout, H, W, hidden=hidden, n_layers=2, seed=1)
    w1 = rng.integers(-64, 65, size=(hidden, cin, 3, 3)) / 64.0
    b1 = rng.integers(-64, 65, size=hidden) / 64.0
    w2 = np.zeros((cout, hidden, 3, 3))
    for j in range(cout):
        w2[j, j, 1, 1] = 1.0
    p = np.concatenate([w1.ravel(), b1, w2.ravel(), np.zeros(cout)]).astype(np.float32)
    assert p.size == net.num_params
    net.set_params(p)
    x = (rng.integers(0, 64, size=(cin, H, W)) / 16.0).astype(np.float32)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    xp = np.pad(x.astype(np.float64), ((0, 0), (1, 1), (1, 1)))
    z = np.zeros((hidden, H, W))
    for dy in range(3):
        for dx in range(3):
            z += np.einsum("oc,chw->ohw", w1[:, :, dy, dx], xp[:, dy:dy + H, dx:dx + W])
    z += b1[:, None, None]
    want = _bf16_round(np.maximum(z, 0.0).astype(np.float32))[:cout]
    assert np.array_equal(y.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [
    dict(),  # one partial tile of 128 positions
    dict(H=9, W=40, cin=80, cout=3, hidden=16, layers=2),  # first layer too wide for the tensor-core tile: GEMM path
])
def test_forward_matches_reference(cuda, shape):
    import torch

    net, x, _ = _net_case(**shape)
    p = net.get_params()
    p[-net.out_channels:] = 0.25  # a nonzero bias somewhere
    net.set_params(p)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref, _ = cnnref.forward(p, net.layer_shapes(), x)
    np.testing.assert_allclose(y, ref, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [
    dict(),  # two position ranges of one 64-position stage each
    dict(H=200, W=200, cin=20, cout=10, hidden=16, layers=3),  # 3 stages per range: both buffers reused
])
def test_gradients_match_reference(cuda, shape):
    import torch

    net, x, t = _net_case(seed=5, **shape)
    p = net.get_params()
    loss, g = net.grads(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    rloss, rg = cnnref.grads(p, net.layer_shapes(), x, t)
    assert loss == pytest.approx(rloss, rel=1e-4)
    np.testing.assert_allclose(g, rg, rtol=2e-3, atol=2e-5 * np.abs(rg).max())


@pytest.mark.gpu
def test_training_reduces_loss(cuda):
    import torch

    net, x, t = _net_case(seed=7, H=24, W=20)
    dx, dt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    first = net.train_step(dx, dt, lr=3e-3)
    for _ in range(150):
        last = net.train_step(dx, dt, lr=3e-3)
    assert last < 0.5 * first
