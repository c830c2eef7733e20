"""CPU oracle of the MSLD lambda maps and biases (src/msld/msld.cu:863-1153)."""
import numpy as np
import pytest

import oracle

BOUND = np.array([0, 1, 4, 8, 11], np.int32)
SITE = np.array([0, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3], np.int32)


def test_lambda_simplex():
    rng = np.random.default_rng(0)
    th = rng.uniform(-2, 2, 11)
    lam = oracle.lambda_from_theta(BOUND, 5.5, th)
    for s in range(len(BOUND) - 1):
        assert lam[BOUND[s]:BOUND[s + 1]].sum() == pytest.approx(1.0, abs=1e-14)
    assert (lam > 0).all()


def test_theta_force_is_chain_rule():
    """dU/dtheta from dU/dlambda equals the FD derivative of U(lambda(theta)) for linear U."""
    rng = np.random.default_rng(1)
    th = rng.uniform(-2, 2, 11)
    F = rng.normal(size=11)                  # U = sum F_b lambda_b
    lam = oracle.lambda_from_theta(BOUND, 5.5, th)
    tf = oracle.theta_force(SITE, BOUND, 5.5, lam, th, F)
    h = 1e-6
    for b in range(1, 11):
        tp = th.copy(); tp[b] += h
        tm = th.copy(); tm[b] -= h
        fd = (F @ oracle.lambda_from_theta(BOUND, 5.5, tp) - F @ oracle.lambda_from_theta(BOUND, 5.5, tm)) / (2 * h)
        assert tf[b] == pytest.approx(fd, rel=1e-6, abs=1e-9)


def test_fixed_block_keeps_theta():
    th = np.array([0.0, 0.3, -0.2, 0.25, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7])
    fixed = np.zeros(11, np.int32)
    fixed[3] = 1
    lam = oracle.lambda_from_theta(BOUND, 5.5, th, fixed)
    assert lam[3] == 0.25
    assert lam[1:4].sum() == pytest.approx(1.0)


@pytest.mark.parametrize("btype,l0,n", [(6, 0.0, 0), (8, 0.017, 0), (10, -5.56, 0), (1, 0.8, 2), (2, 0.2, 2),
                                         (3, 0.0, 2), (4, 0.5, 0), (5, 0.0, 0), (7, 0.1, 0), (11, 2.0, 2), (12, 0.1, 2)])
def test_bias_fd(btype, l0, n):
    lam = np.array([1.0, 0.3, 0.6, 0.1])
    vb = np.zeros(1, oracle.VARBIAS_DTYPE)
    vb[0] = (1, 2, btype, l0, 3.5, n)
    fixed = np.array([0.0, 1.5, -2.0, 0.7])
    lf, e = oracle.bias(lam, fixed, vb)
    h = 1e-7
    for b in (1, 2):
        lp = lam.copy(); lp[b] += h
        lm = lam.copy(); lm[b] -= h
        fd = (oracle.bias(lp, fixed, vb)[1] - oracle.bias(lm, fixed, vb)[1]) / (2 * h)
        assert lf[b] == pytest.approx(fd, rel=1e-5, abs=1e-6)
