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


@pytest.mark.gpu
def test_forward_matches_reference(cuda):
    import torch

    net, x, _ = _net_case()
    p = net.get_params()
    p[-net.out_channels:] = 0.25  # a nonzero bias somewhere
    net.set_params(p)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref, _ = cnnref.forward(p, net.layer_shapes(), x)
    np.testing.assert_allclose(y, ref, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_gradients_match_reference(cuda):
    import torch

    net, x, t = _net_case(seed=5)
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
