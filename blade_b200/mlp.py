"""BF16 MLP trained and run with libbnb's own kernels (csrc/mlp.cu).

Used by learned landscape flattening (``blade_b200.alf``): 3 hidden layers of
256 with SiLU, BF16 weights and activations, FP32 accumulation, FP32 master
weights updated by Adam.  torch provides device memory and the stream only;
every forward, backward, loss and optimizer step is a libbnb kernel.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class BF16MLP:
    def __init__(self, sizes, max_batch: int, seed: int = 0, device="cuda"):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.sizes = list(sizes)
        self.max_batch = max_batch
        rng = np.random.default_rng(seed)
        f32, bf = torch.float32, torch.int16
        self.W, self.Wb, self.b, self.mW, self.vW, self.mb, self.vb, self.gW, self.gb = ([] for _ in range(9))
        for K, N in zip(self.sizes[:-1], self.sizes[1:]):
            bound = np.sqrt(6.0 / K) if len(self.W) < len(self.sizes) - 2 else np.sqrt(1.0 / K)
            w = rng.uniform(-bound, bound, (N, K)).astype(np.float32)
            self.W.append(torch.from_numpy(w).to(self.dev))
            self.Wb.append(torch.empty(N * K, dtype=bf, device=self.dev))
            self.b.append(torch.zeros(N, dtype=f32, device=self.dev))
            for lst, n in ((self.mW, N * K), (self.vW, N * K), (self.gW, N * K), (self.mb, N), (self.vb, N),
                           (self.gb, N)):
                lst.append(torch.zeros(n, dtype=f32, device=self.dev))
        self._sync_bf16()
        M = max_batch
        self.xb = torch.empty(M * self.sizes[0], dtype=bf, device=self.dev)
        self.Z = [torch.empty(M * n, dtype=f32, device=self.dev) for n in self.sizes[1:]]
        self.Yb = [torch.empty(M * n, dtype=bf, device=self.dev) for n in self.sizes[1:-1]]
        self.out = torch.empty(M * self.sizes[-1], dtype=f32, device=self.dev)
        self.dY = [torch.empty(M * n, dtype=f32, device=self.dev) for n in self.sizes[1:]]
        self.dZ = [torch.empty(M * n, dtype=f32, device=self.dev) for n in self.sizes[1:]]
        self.dZb = [torch.empty(M * n, dtype=bf, device=self.dev) for n in self.sizes[1:]]
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.step_count = 0

    # -- helpers -------------------------------------------------------------------
    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _sync_bf16(self):
        for W, Wb in zip(self.W, self.Wb):
            _lib.call("bnb_to_bf16", W.numel(), _p(W), _p(Wb), self._s())

    @property
    def n_layers(self):
        return len(self.W)

    # -- forward / backward ----------------------------------------------------------
    def forward(self, x):
        """x: device FP32 [M, sizes[0]] -> device FP32 [M, sizes[-1]] (a view of an internal buffer)."""
        M = x.shape[0]
        assert M <= self.max_batch and x.shape[1] == self.sizes[0] and x.dtype == self.torch.float32
        s = self._s()
        _lib.call("bnb_to_bf16", M * self.sizes[0], _p(x.contiguous()), _p(self.xb), s)
        h = self.xb
        for l in range(self.n_layers):
            K, N = self.sizes[l], self.sizes[l + 1]
            last = l == self.n_layers - 1
            _lib.call("bnb_mlp_linear_forward", M, N, K, _p(h), _p(self.Wb[l]), _p(self.b[l]), 0 if last else 1,
                      _p(self.Z[l]), None if last else _p(self.Yb[l]), _p(self.out) if last else None, s)
            if not last:
                h = self.Yb[l]
        return self.out[:M * self.sizes[-1]].view(M, self.sizes[-1])

    def backward(self, M: int, dout):
        """dout: device FP32 [M, sizes[-1]] = dLoss/dOutput; fills gW, gb."""
        s = self._s()
        dy = dout
        for l in range(self.n_layers - 1, -1, -1):
            K, N = self.sizes[l], self.sizes[l + 1]
            x_in = self.xb if l == 0 else self.Yb[l - 1]
            dx = None if l == 0 else self.dY[l - 1]
            _lib.call("bnb_mlp_linear_backward", M, N, K, _p(dy), _p(self.Z[l]), 0 if l == self.n_layers - 1 else 1,
                      _p(x_in), _p(self.Wb[l]), _p(self.dZ[l]), _p(self.dZb[l]), _p(dx), _p(self.gW[l]),
                      _p(self.gb[l]), s)
            dy = dx

    def loss_grad(self, x, target, weight=None, elem_weight=None):
        """Forward + MSE + backward; returns the device loss tensor (FP64 [1]).
        weight: per output column [N]; elem_weight: per element [M, N]."""
        M = x.shape[0]
        out = self.forward(x)
        dout = self.dY[-1]
        ew = None if elem_weight is None else elem_weight.contiguous()
        _lib.call("bnb_mlp_mse", M, self.sizes[-1], _p(out), _p(target.contiguous()), _p(weight), _p(ew),
                  _p(dout), _p(self.loss), self._s())
        self.backward(M, dout)
        return self.loss

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.step_count += 1
        s = self._s()
        for l in range(self.n_layers):
            _lib.call("bnb_mlp_adam", self.W[l].numel(), _p(self.W[l]), _p(self.Wb[l]), _p(self.gW[l]),
                      _p(self.mW[l]), _p(self.vW[l]), lr, beta1, beta2, eps, weight_decay, self.step_count, s)
            _lib.call("bnb_mlp_adam", self.b[l].numel(), _p(self.b[l]), None, _p(self.gb[l]), _p(self.mb[l]),
                      _p(self.vb[l]), lr, beta1, beta2, eps, 0.0, self.step_count, s)

    def train_step(self, x, target, weight=None, lr=1e-3, elem_weight=None):
        loss = self.loss_grad(x, target, weight, elem_weight)
        self.adam_step(lr)
        return loss

    # -- state -----------------------------------------------------------------------
    def state(self) -> dict:
        d = {"sizes": np.array(self.sizes)}
        for l in range(self.n_layers):
            d[f"W{l}"] = self.W[l].cpu().numpy()
            d[f"b{l}"] = self.b[l].cpu().numpy()
        return d

    def load(self, d: dict):
        """Weights from ``state()``, or from a file that stores each weight
        matrix as its BF16 bit patterns (``W{l}_bf16``)."""
        d = weights_from_file_dict(d)
        assert list(d["sizes"]) == self.sizes
        for l in range(self.n_layers):
            self.W[l].copy_(self.torch.from_numpy(np.asarray(d[f"W{l}"], np.float32)))
            self.b[l].copy_(self.torch.from_numpy(np.asarray(d[f"b{l}"], np.float32)))
        self._sync_bf16()


def weights_from_file_dict(d: dict) -> dict:
    """``W{l}`` FP32 from ``W{l}_bf16`` (uint16 BF16 bit patterns) where only
    the latter is present; other entries unchanged."""
    out = dict(d)
    l = 0
    while f"W{l}_bf16" in out or f"W{l}" in out:
        if f"W{l}" not in out:
            bits = np.asarray(out[f"W{l}_bf16"], np.uint16).astype(np.uint32) << 16
            out[f"W{l}"] = bits.view(np.float32)
        l += 1
    return out
