"""Congestion lookahead: a small convolutional network over the routing grid.

The network (``gr_cnn_*`` in the C ABI) reads, per routing layer, the
current demand and capacity of every GCELL and predicts the demand the
remaining batches will still add. It is trained on snapshots of the router's
own runs (demand after 10/25/50/75 % of the batches against the final
demand) and its prediction becomes a lookahead term of the GCELL cost used
by the L-pattern stage.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import check, lib, ptr


class LookaheadNet:
    """``n_layers`` 3x3 convolutions, ``hidden`` channels, ReLU between layers.

    Inputs and outputs are CUDA float32 tensors of shape (channels, H, W).
    Parameters per layer: weights (cout, cin, 3, 3) then biases (cout,).
    """

    def __init__(self, in_channels: int, out_channels: int, H: int, W: int, hidden: int = 32, n_layers: int = 4,
                 seed: int = 1, device: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        check(self._lib.gr_cnn_create(C.byref(h), device, in_channels, out_channels, hidden, n_layers, H, W, seed),
              "gr_cnn_create")
        self._h = h
        self.in_channels, self.out_channels, self.H, self.W = in_channels, out_channels, H, W
        self.hidden, self.n_layers, self.device = hidden, n_layers, device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gr_cnn_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def num_params(self) -> int:
        return int(self._lib.gr_cnn_num_params(self._h))

    def layer_shapes(self):
        """[(cin, cout)] per layer."""
        out = []
        for l in range(self.n_layers):
            cin = self.in_channels if l == 0 else self.hidden
            cout = self.out_channels if l + 1 == self.n_layers else self.hidden
            out.append((cin, cout))
        return out

    def get_params(self) -> np.ndarray:
        out = np.empty(self.num_params, dtype=np.float32)
        check(self._lib.gr_cnn_get_params(self._h, ptr(out)), "gr_cnn_get_params")
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params
        check(self._lib.gr_cnn_set_params(self._h, ptr(p)), "gr_cnn_set_params")

    def _check_in(self, x):
        assert x.is_cuda and x.dtype.is_floating_point and x.is_contiguous()
        assert tuple(x.shape) == (self.in_channels, self.H, self.W), x.shape

    def forward(self, x):
        import torch

        self._check_in(x)
        y = torch.empty((self.out_channels, self.H, self.W), dtype=torch.float32, device=x.device)
        check(self._lib.gr_cnn_forward(self._h, x.data_ptr(), y.data_ptr()), "gr_cnn_forward")
        return y

    def grads(self, x, target):
        """(loss, gradients in parameter layout) of the mean squared error."""
        self._check_in(x)
        g = np.empty(self.num_params, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        check(self._lib.gr_cnn_grads(self._h, x.data_ptr(), target.data_ptr(), ptr(g), ptr(loss)), "gr_cnn_grads")
        return float(loss[0]), g

    def train_step(self, x, target, lr: float = 1e-3) -> float:
        self._check_in(x)
        loss = np.zeros(1, dtype=np.float32)
        check(self._lib.gr_cnn_train_step(self._h, x.data_ptr(), target.data_ptr(), C.c_float(lr), ptr(loss)),
              "gr_cnn_train_step")
        return float(loss[0])
