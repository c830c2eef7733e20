"""BF16 MLP kernels (csrc/mlp.cu) against the FP64 CPU oracle
(oracle/mlp_oracle.py): layer by layer on the kernels' own BF16 operands
(only FP32-vs-FP64 accumulation differs), the whole network end to end, the
Adam step, and a training run that must reduce the loss."""
import ctypes as C

import numpy as np
import pytest
import torch

from blade_b200 import _lib
from blade_b200.mlp import BF16MLP
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

ACC_TOL = 2e-5      # max |gpu - oracle| / max |oracle|, same BF16 operands
E2E_TOL = 1e-2      # relative L2 of whole-network gradients (BF16 rounding may flip)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _bf16(x):
    x = torch.as_tensor(np.ascontiguousarray(x, np.float32), device="cuda")
    y = torch.empty(x.numel(), dtype=torch.int16, device="cuda")
    _lib.call("bnb_to_bf16", x.numel(), _p(x), _p(y), _s())
    return y


def _decode(t, shape):
    return mo.from_bf16_bits(t.cpu().numpy().view(np.uint16)).reshape(shape)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("act", [0, 1])
def test_linear_forward_backward_match_oracle(cuda, act):
    rng = np.random.default_rng(act)
    M, K, N = 96, 200, 130
    X = _bf16(rng.normal(size=(M, K)))
    W = _bf16(rng.normal(0, 0.1, (N, K)))
    b = torch.as_tensor(rng.normal(0, 0.1, N).astype(np.float32), device="cuda")
    Z = torch.empty(M * N, device="cuda")
    Yb = torch.empty(M * N, dtype=torch.int16, device="cuda")
    Yf = torch.empty(M * N, device="cuda")
    _lib.call("bnb_mlp_linear_forward", M, N, K, _p(X), _p(W), _p(b), act, _p(Z), _p(Yb), _p(Yf), _s())
    Xh, Wh = _decode(X, (M, K)), _decode(W, (N, K))
    Zo, Yo = mo.linear_forward(Xh, Wh, b.cpu().numpy().astype(np.float64), act)
    assert _rel(Z.cpu().numpy().reshape(M, N), Zo) < ACC_TOL
    assert _rel(Yf.cpu().numpy().reshape(M, N), Yo) < ACC_TOL
    # BF16 output is the FP32 output rounded to nearest even
    np.testing.assert_array_equal(_decode(Yb, (M, N)), mo.bf16_round(Yf.cpu().numpy().reshape(M, N)))

    dY = torch.as_tensor(rng.normal(size=(M, N)).astype(np.float32), device="cuda")
    dZ = torch.empty(M * N, device="cuda")
    dZb = torch.empty(M * N, dtype=torch.int16, device="cuda")
    dX = torch.empty(M * K, device="cuda")
    dW = torch.empty(N * K, device="cuda")
    db = torch.empty(N, device="cuda")
    _lib.call("bnb_mlp_linear_backward", M, N, K, _p(dY), _p(Z), act, _p(X), _p(W), _p(dZ), _p(dZb), _p(dX),
              _p(dW), _p(db), _s())
    Zg = Z.cpu().numpy().reshape(M, N).astype(np.float64)
    dZo, _, _, _, dbo = mo.linear_backward(dY.cpu().numpy().astype(np.float64), Zg, act, Xh, Wh)
    assert _rel(dZ.cpu().numpy().reshape(M, N), dZo) < ACC_TOL
    assert _rel(db.cpu().numpy(), dbo) < ACC_TOL
    dZh = _decode(dZb, (M, N))
    np.testing.assert_array_equal(dZh, mo.bf16_round(dZ.cpu().numpy().reshape(M, N)))
    assert _rel(dW.cpu().numpy().reshape(N, K), dZh.T @ Xh) < ACC_TOL
    assert _rel(dX.cpu().numpy().reshape(M, K), dZh @ Wh) < ACC_TOL


def test_network_gradients_match_oracle(cuda):
    rng = np.random.default_rng(5)
    sizes = [72, 64, 64, 40]
    net = BF16MLP(sizes, max_batch=48, seed=3)
    x = rng.normal(size=(48, 72)).astype(np.float32)
    t = rng.normal(size=(48, 40)).astype(np.float32)
    w = rng.uniform(0.5, 1.5, 40).astype(np.float32)
    loss = net.loss_grad(torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda"),
                         torch.as_tensor(w, device="cuda"))
    st = net.state()
    Ws = [st[f"W{l}"].astype(np.float64) for l in range(3)]
    bs = [st[f"b{l}"].astype(np.float64) for l in range(3)]
    lo, go = mo.mlp_loss_grad(x.astype(np.float64), t.astype(np.float64), Ws, bs, w.astype(np.float64))
    assert abs(float(loss.cpu()[0]) - lo) <= 1e-3 * lo
    for l in range(3):
        gW = net.gW[l].cpu().numpy().reshape(go[l][0].shape)
        gb = net.gb[l].cpu().numpy()
        assert np.linalg.norm(gW - go[l][0]) <= E2E_TOL * np.linalg.norm(go[l][0])
        assert np.linalg.norm(gb - go[l][1]) <= E2E_TOL * np.linalg.norm(go[l][1])


def test_adam_matches_oracle(cuda):
    rng = np.random.default_rng(9)
    n = 1000
    w0 = rng.normal(size=n).astype(np.float32)
    g = rng.normal(size=n).astype(np.float32)
    m0 = rng.normal(0, 0.1, n).astype(np.float32)
    v0 = rng.uniform(0, 0.1, n).astype(np.float32)
    W, G, Mm, V = (torch.as_tensor(a.copy(), device="cuda") for a in (w0, g, m0, v0))
    Wb = torch.empty(n, dtype=torch.int16, device="cuda")
    _lib.call("bnb_mlp_adam", n, _p(W), _p(Wb), _p(G), _p(Mm), _p(V), 1e-3, 0.9, 0.999, 1e-8, 1e-2, 7, _s())
    wo, mo_, vo = mo.adam(w0.astype(np.float64), g.astype(np.float64), m0.astype(np.float64),
                          v0.astype(np.float64), 1e-3, 0.9, 0.999, 1e-8, 1e-2, 7)
    np.testing.assert_allclose(W.cpu().numpy(), wo, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(Mm.cpu().numpy(), mo_, rtol=1e-5, atol=1e-7)
    np.testing.assert_array_equal(_decode(Wb, (n,)), mo.bf16_round(W.cpu().numpy()))


def test_training_reduces_loss(cuda):
    rng = np.random.default_rng(11)
    A = rng.normal(0, 0.3, (16, 64))
    x = rng.normal(size=(512, 64)).astype(np.float32)
    t = np.tanh(x @ A.T).astype(np.float32)
    net = BF16MLP([64, 128, 128, 16], max_batch=128, seed=1)
    X = torch.as_tensor(x, device="cuda")
    T = torch.as_tensor(t, device="cuda")
    first = float(net.loss_grad(X[:128], T[:128]).cpu()[0])
    for it in range(300):
        k = (it % 4) * 128
        net.train_step(X[k:k + 128], T[k:k + 128], lr=3e-3)
    last = float(net.loss_grad(X[:128], T[:128]).cpu()[0])
    assert last < 0.1 * first
