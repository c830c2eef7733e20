"""GPU pieces of landscape flattening: the lambda histogram kernel against
numpy, and the ALF bias terms in the batched step against the oracle's FP64
bias routine."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from blade_b200 import _lib, alf, systems
from blade_b200.batch import MsldBatch

pytestmark = pytest.mark.gpu


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def test_lambda_histogram_kernel(cuda):
    rng = np.random.default_rng(0)
    L, P, steps = 40, 25, 7
    fixed = np.zeros(L, np.uint8)
    fixed[[0, 13]] = 1
    pairs = rng.integers(0, L, (P, 2)).astype(np.int32)
    h1 = torch.zeros(L * 32, dtype=torch.int32, device="cuda")
    h2 = torch.zeros(P * 64, dtype=torch.int32, device="cuda")
    he = torch.zeros(L, dtype=torch.int32, device="cuda")
    fx = torch.as_tensor(fixed, device="cuda")
    pr = torch.as_tensor(pairs.reshape(-1), device="cuda")
    e1, e2, ee = np.zeros((L, 32), np.int64), np.zeros((P, 8, 8), np.int64), np.zeros(L, np.int64)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for k in range(steps):
        lam = rng.uniform(0, 1, L)
        lam[:5] = [0.0, 1.0, 0.99, 0.990001, 0.5]
        lt = torch.as_tensor(lam, device="cuda")
        _lib.call("bnb_lambda_histogram", L, _p(lt), _p(fx), P, _p(pr), _p(h1), _p(h2), _p(he), s)
        b = np.minimum((lam * 32).astype(int), 31)
        for i in range(L):
            if not fixed[i]:
                e1[i, b[i]] += 1
                ee[i] += lam[i] > 0.99
        for p, (i, j) in enumerate(pairs):
            e2[p, min(int(lam[i] * 8), 7), min(int(lam[j] * 8), 7)] += 1
    np.testing.assert_array_equal(h1.cpu().numpy().reshape(L, 32), e1)
    np.testing.assert_array_equal(h2.cpu().numpy().reshape(P, 8, 8), e2)
    np.testing.assert_array_equal(he.cpu().numpy(), ee)


def test_batch_bias_matches_oracle(cuda):
    reps = [systems.msld_water(100 + k, avoid_sites=True, charge_sigma=0.15) for k in range(2)]
    B = MsldBatch(reps, T=0.0)
    sm = alf.site_map(reps, B.nb.lam_starts)
    params = np.random.default_rng(2).normal(0, 3, sm.n_params)
    fixed, var = alf.bias_arrays(sm, params)
    B.set_bias(fixed, var)
    lam = B.lam.cpu().numpy()
    lf = torch.zeros_like(B.lforce)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.call("bnb_bias", B.theta.numel(), _p(B.lam), _p(B.fixed_bias), B.n_var, _p(B.var_bias), _p(lf), None, s)
    lo, _ = oracle.bias(lam, fixed, var)
    np.testing.assert_allclose(lf.cpu().numpy(), lo, rtol=1e-6, atol=1e-6)
    B.close()


def test_gpu_histograms_equal_trajectory_histograms(cuda):
    """Histograms accumulated on the GPU during stepping equal those built
    from the lambda trajectory of the same steps (what ALF reads from .lmd)."""
    from blade_b200 import lmd
    reps = [alf.flattening_system(100 + k) for k in range(2)]
    B = MsldBatch(reps, gamma_ps=5.0, theta_mass=5.0, gamma_theta_ps=1.0)
    sm = alf.site_map(reps, B.nb.lam_starts)
    B.enable_histograms(sm.pairs)
    traj = []
    for k in range(40):
        B.enqueue_step(k)
        traj.append(B.lam.cpu().numpy().copy())
    h1, h2, he = B.take_histograms()
    r1, r2, re = lmd.histograms(np.array(traj), sm.pairs, B.fixed.cpu().numpy().astype(bool))
    np.testing.assert_array_equal(h1, r1)
    np.testing.assert_array_equal(h2, r2)
    np.testing.assert_array_equal(he, re)
    B.close()
