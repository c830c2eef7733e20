"""FP64 CPU restatement of the BF16 MLP kernels (test infrastructure only).

This is the checker for blade_b200/csrc/mlp.cu: the same layer algebra in
numpy FP64, with BF16 rounding (round to nearest even) applied at the same
points as the kernels -- operands of every product (inputs X, weights W,
hidden activations Y, the backward's dZ) -- so that the only remaining
difference is the kernels' FP32 accumulation.  The network has no reference
counterpart (BLaDE's src/mlp is unrelated TorchANI inference); parity of the
flattening algebra itself is unpinned against ALF, which is not in the
reference tree.  Only tests/ and the measurement scripts import this module.
"""
from __future__ import annotations

import numpy as np


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    nan = np.isnan(f)
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    out[nan] = np.nan
    return out


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """BF16 bit patterns (uint16) of bf16_round(x)."""
    return (bf16_round(x).astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def linear_forward(X, W, b, act: int):
    """X [M,K], W [N,K] (already BF16 values), b [N] -> (Z, Y) in FP64.
    Z = X W^T + b; Y = act(Z) (the BF16 copy is bf16_round(Y))."""
    Z = X @ W.T + (0.0 if b is None else b)
    Y = silu(Z) if act else Z
    return Z, Y


def linear_backward(dY, Z, act: int, X, W):
    """Returns (dZ, dZb, dX, dW, db): dZb = bf16(dZ) is the products' operand."""
    dZ = dY * silu_grad(Z) if act else dY.copy()
    dZb = bf16_round(dZ)
    return dZ, dZb, dZb @ W, dZb.T @ X, dZ.sum(0)


def mse(Y, T, w=None, we=None):
    M = Y.shape[0]
    w = np.ones(Y.shape[1]) if w is None else w
    if we is not None:
        w = w * we
    d = Y - T
    return float((w * d * d).sum() / M), 2.0 * w * d / M


def mlp_forward(x, weights, biases, round_bf16=True):
    """Whole network (SiLU on all but the last layer).  Returns the list of
    layer inputs (as BF16 values) and the per-layer (Z, Y)."""
    rnd = bf16_round if round_bf16 else (lambda a: np.asarray(a, np.float64))
    inputs, outs = [], []
    h = rnd(x)
    for l, (W, b) in enumerate(zip(weights, biases)):
        act = 1 if l < len(weights) - 1 else 0
        inputs.append(h)
        Z, Y = linear_forward(h, rnd(W), b, act)
        outs.append((Z, Y))
        h = rnd(Y)
    return inputs, outs


def mlp_loss_grad(x, t, weights, biases, w=None, round_bf16=True):
    """Loss and gradients (dW, db per layer) of the MSE of the last layer's FP32 output."""
    rnd = bf16_round if round_bf16 else (lambda a: np.asarray(a, np.float64))
    inputs, outs = mlp_forward(x, weights, biases, round_bf16)
    loss, dY = mse(outs[-1][1], t, w)
    grads = [None] * len(weights)
    for l in range(len(weights) - 1, -1, -1):
        act = 1 if l < len(weights) - 1 else 0
        dZ = dY * silu_grad(outs[l][0]) if act else dY
        dZb = rnd(dZ)
        grads[l] = (dZb.T @ inputs[l], dZ.sum(0))
        dY = dZb @ rnd(weights[l])
    return loss, grads


def adam(master, g, m, v, lr, b1, b2, eps, wd, step):
    """One Adam step in FP64 (the kernel's order of operations)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    master = master - lr * ((m / c1) / (np.sqrt(v / c2) + eps) + wd * master)
    return master, m, v
