"""CPU checks of the FP64 MLP oracle: BF16 rounding and its backward pass
against central finite differences (without rounding, so the derivative is
that of a smooth function)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_round_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e-39, 65504.0], np.float32)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7 -> even (1); 1 + 3*2^-8 -> 1 + 2^-6
    np.testing.assert_array_equal(mo.bf16_round(x)[:3], [1.0, 1.0, 1.015625])
    assert mo.bf16_round(np.float32([-2.5]))[0] == -2.5
    b = mo.bf16_bits(np.float32([1.0, -2.0]))
    assert b.tolist() == [0x3F80, 0xC000]
    np.testing.assert_array_equal(mo.from_bf16_bits(b), [1.0, -2.0])


def _net(rng, sizes):
    Ws = [rng.normal(0, 1 / np.sqrt(k), (n, k)) for k, n in zip(sizes[:-1], sizes[1:])]
    bs = [rng.normal(0, 0.1, n) for n in sizes[1:]]
    return Ws, bs


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    sizes = [7, 6, 5, 3]
    Ws, bs = _net(rng, sizes)
    x = rng.normal(size=(4, 7))
    t = rng.normal(size=(4, 3))
    w = np.array([1.0, 0.5, 2.0])
    loss, grads = mo.mlp_loss_grad(x, t, Ws, bs, w, round_bf16=False)
    h = 1e-6
    for l in range(len(Ws)):
        for (i, j) in [(0, 0), (1, 2), (Ws[l].shape[0] - 1, Ws[l].shape[1] - 1)]:
            Wp = [W.copy() for W in Ws]
            Wm = [W.copy() for W in Ws]
            Wp[l][i, j] += h
            Wm[l][i, j] -= h
            fd = (mo.mlp_loss_grad(x, t, Wp, bs, w, False)[0] - mo.mlp_loss_grad(x, t, Wm, bs, w, False)[0]) / (2 * h)
            assert abs(fd - grads[l][0][i, j]) < 1e-6 * max(1.0, abs(fd))
        for i in range(bs[l].shape[0]):
            bp = [b.copy() for b in bs]
            bm = [b.copy() for b in bs]
            bp[l][i] += h
            bm[l][i] -= h
            fd = (mo.mlp_loss_grad(x, t, Ws, bp, w, False)[0] - mo.mlp_loss_grad(x, t, Ws, bm, w, False)[0]) / (2 * h)
            assert abs(fd - grads[l][1][i]) < 1e-6 * max(1.0, abs(fd))


def test_adam_first_step_moves_by_lr():
    m0 = np.zeros(3)
    w, m, v = mo.adam(np.ones(3), np.array([0.5, -2.0, 1e-3]), m0, m0, 0.01, 0.9, 0.999, 1e-12, 0.0, 1)
    np.testing.assert_allclose(w, [0.99, 1.01, 0.99], rtol=1e-9)
