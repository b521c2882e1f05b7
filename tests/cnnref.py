"""Float64 NumPy restatement of the lookahead network (test infrastructure).

It rounds every GEMM operand to BF16 exactly as the CUDA kernels do (the
im2col columns, the packed weights and the activation gradients), so the
CUDA results differ from it only by the FP32 accumulation order of the
tensor-core GEMMs."""
import numpy as np


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(x):
    """Round to float32, as float64 (the kernels' FP32 intermediates)."""
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def q(x):
    """A GEMM operand: float32, then BF16."""
    return bf16(np.asarray(x, dtype=np.float32))


def im2col(x):
    """x (cin, H, W) -> (H*W, cin*9), column k = ci*9 + (dy+1)*3 + (dx+1), zero padding."""
    cin, H, W = x.shape
    p = np.zeros((cin, H + 2, W + 2))
    p[:, 1:-1, 1:-1] = x
    cols = np.empty((H * W, cin * 9))
    for r in range(9):
        dy, dx = r // 3, r % 3
        cols[:, r::9] = p[:, dy:dy + H, dx:dx + W].reshape(cin, H * W).T
    return cols


def col2im(dcol, cin, H, W):
    """Adjoint of im2col."""
    p = np.zeros((cin, H + 2, W + 2))
    for r in range(9):
        dy, dx = r // 3, r % 3
        p[:, dy:dy + H, dx:dx + W] += dcol[:, r::9].T.reshape(cin, H, W)
    return p[:, 1:-1, 1:-1]


def split(params, shapes):
    out, o = [], 0
    for cin, cout in shapes:
        w = params[o:o + cout * cin * 9].reshape(cout, cin * 9).astype(np.float64)
        o += cout * cin * 9
        b = params[o:o + cout].astype(np.float64)
        o += cout
        out.append((w, b))
    return out


def forward(params, shapes, x):
    """Returns (output (cout, H, W), per-layer (input, pre-activation (M, cout)))."""
    _, H, W = x.shape
    a = np.asarray(x, dtype=np.float64)
    saved = []
    for l, (w, b) in enumerate(split(params, shapes)):
        col = q(im2col(a))
        pre = col @ q(w).T + b
        saved.append((a, pre))
        y = np.maximum(pre, 0) if l + 1 < len(shapes) else pre
        a = y.T.reshape(w.shape[0], H, W)
    return a, saved


def grads(params, shapes, x, target):
    """(loss, gradient in parameter layout) of the mean squared error."""
    _, H, W = x.shape
    y, saved = forward(params, shapes, x)
    t = np.asarray(target, dtype=np.float64)
    n = y.size
    loss = float(((y - t) ** 2).sum() / n)
    dy = f32(2.0 * (y - t) / n)
    layers = split(params, shapes)
    g = []
    for l in range(len(shapes) - 1, -1, -1):
        (w, b), (a, pre) = layers[l], saved[l]
        cout = w.shape[0]
        dz = dy.reshape(cout, H * W).T.copy()
        if l + 1 < len(shapes):
            dz[pre <= 0] = 0.0
        dzb = q(dz)
        col = q(im2col(a))
        gw = (col.T @ dzb).T
        gb = dzb.sum(axis=0)
        g.append(np.concatenate([gw.ravel(), gb]))
        if l > 0:
            dcol = dzb @ q(w)
            dy = f32(col2im(dcol, a.shape[0], H, W))
    return loss, np.concatenate(g[::-1])
