"""Holonomic constraints on the GPU (bnb_holonomic_position /
bnb_holonomic_velocity) against the FP64 oracle and the reference's golden
vectors; the split Langevin step against the fused one; and the batched MSLD
step with rigid waters."""
import glob
import os

import numpy as np
import pytest
import torch

from blade_b200 import _lib, systems
from blade_b200.holonomic import Constraints
from oracle import holonomic_oracle as H

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64).reshape(-1)).cuda()


@pytest.mark.parametrize("jitter", [0.01, 0.05])
def test_position_matches_oracle(cuda, jitter):
    T, B1, B2, B3, xp, x, ism = H.test_clusters(seed=5, jitter=jitter)
    cs = Constraints(T, B1, B2, B3)
    xg, vg, st = _t(x), torch.zeros(x.size, dtype=torch.float64, device="cuda"), torch.zeros(1, dtype=torch.int32,
                                                                                             device="cuda")
    xf = torch.zeros(x.size, dtype=torch.float32, device="cuda")
    cs.position(_t(xp), xg, vg, _t(ism), 0.02, tolerance=1e-12, max_iter=20, x_f=xf, status=st)
    xo, vo, _ = H.constrain_position(H.clusters(T, B1, B2, B3), xp, x, ism, 0.02)
    assert int(st.item()) == 0
    assert np.abs(xg.cpu().numpy().reshape(-1, 3) - xo).max() < 1e-10
    assert np.abs(vg.cpu().numpy().reshape(-1, 3) - vo).max() < 1e-8
    assert torch.equal(xf, xg.float())


def test_not_converged_sets_status(cuda):
    T, B1, B2, B3, xp, x, ism = H.test_clusters(seed=5, jitter=0.05)
    cs = Constraints(T, B1, B2, B3)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    cs.position(_t(xp), _t(x), None, _t(ism), 0.02, tolerance=1e-14, max_iter=1, status=st)
    assert int(st.item()) == 1


def test_velocity_matches_oracle(cuda):
    T, B1, B2, B3, xp, x, ism = H.test_clusters(seed=6)
    cs = Constraints(T, B1, B2, B3)
    v0 = np.random.default_rng(1).normal(size=xp.shape)
    vg = _t(v0)
    cs.velocity(_t(xp), vg, _t(ism))
    vo = H.constrain_velocity(H.clusters(T, B1, B2, B3), xp, v0, ism)
    assert np.abs(vg.cpu().numpy().reshape(-1, 3) - vo).max() < 1e-10


GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "holonomic_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(f)[:-4] for f in GOLDEN])
def test_matches_reference_golden(cuda, path):
    z = np.load(path)
    T = z["tri"].view(H.TRI_DTYPE)
    B1, B2, B3 = z["b1"].view(H.B1_DTYPE), z["b2"].view(H.B2_DTYPE), z["b3"].view(H.B3_DTYPE)
    cs = Constraints(T, B1, B2, B3)
    xg, vg = _t(z["x"]), torch.zeros(z["x"].size, dtype=torch.float64, device="cuda")
    cs.position(_t(z["x_prev"]), xg, vg, _t(z["ism"]), float(z["halfdt"]), tolerance=1e-10)
    assert np.abs(xg.cpu().numpy().reshape(-1, 3) - z["x_ref"]).max() < 1e-7
    v = vg.cpu().numpy().reshape(-1, 3)
    assert np.sqrt(((v - z["v_ref"]) ** 2).sum() / (z["v_ref"] ** 2).sum()) < 1e-5


def test_split_step_equals_fused(cuda):
    """bnb_langevin_half phase 0 then 1 gives the bits of bnb_langevin_vrorv."""
    import ctypes as C
    rng = np.random.default_rng(3)
    nx, nt = 3000, 7
    x0, v0, f0 = rng.normal(size=nx), rng.normal(size=nx), rng.normal(size=nx)
    ism = np.abs(rng.normal(size=nx)) + 0.1
    t0, vt0, ft0, ismt = rng.normal(size=nt), rng.normal(size=nt), rng.normal(size=nt), np.full(nt, 0.3)
    P = lambda t: C.c_void_p(t.data_ptr())
    outs = []
    for split in (False, True):
        x, v, th, vt = _t(x0), _t(v0), _t(t0), _t(vt0)
        xf = torch.zeros(nx, dtype=torch.float32, device="cuda")
        args = (P(x), P(v))
        if split:
            xp = torch.zeros(nx, dtype=torch.float64, device="cuda")
            for phase in (0, 1):
                _lib.call("bnb_langevin_half", phase, nx, nt, P(x), P(v), P(xp), P(_t(f0)), P(_t(ism)), P(th), P(vt),
                          P(_t(ft0)), P(_t(ismt)), 0.04, 0.9, 0.3, 0.95, 0.2, C.c_ulonglong(11), C.c_ulonglong(5),
                          None, P(xf), None, None)
        else:
            _lib.call("bnb_langevin_vrorv", nx, nt, *args, P(_t(f0)), P(_t(ism)), P(th), P(vt), P(_t(ft0)),
                      P(_t(ismt)), 0.04, 0.9, 0.3, 0.95, 0.2, C.c_ulonglong(11), C.c_ulonglong(5), None, P(xf),
                      None, None)
        torch.cuda.synchronize()
        outs.append((x.cpu(), v.cpu(), th.cpu(), vt.cpu(), xf.cpu()))
    for a, b in zip(*outs):
        assert torch.equal(a, b)


def test_batch_with_rigid_waters(cuda):
    from blade_b200.batch import MsldBatch
    reps = [systems.msld_chain(41, 3000, 1, [3]), systems.msld_chain(42, 3600, 2, [2, 2])]
    B = MsldBatch(reps, constraints=True)
    B.run_eager(20)
    B.capture()
    B.run_graph(20)
    torch.cuda.synchronize()
    assert int(B.cons_status.item()) == 0
    st, nan = B.check()
    assert st == 0 and nan == 0
    x = B.x.cpu().numpy().reshape(-1, 3)
    tri = B.cons._keep[0][1].cpu().numpy().view(H.TRI_DTYPE)
    d01 = np.linalg.norm(x[tri["idx"][:, 0]] - x[tri["idx"][:, 1]], axis=1)
    d12 = np.linalg.norm(x[tri["idx"][:, 1]] - x[tri["idx"][:, 2]], axis=1)
    assert np.abs(d01 - 0.9572).max() < 1e-6 and np.abs(d12 - 1.5139).max() < 1e-6
    B.close()


def test_empty_and_single_cluster_types(cuda):
    """Each cluster type alone, and an empty set (no launch)."""
    T, B1, B2, B3, xp, x, ism = H.test_clusters(seed=8, n_water=3, n_each=2, jitter=0.02)
    for sets in ((T, None, None, None), (None, B1, None, None), (None, None, B2, None), (None, None, None, B3)):
        cs = Constraints(*sets)
        xg = _t(x)
        cs.position(_t(xp), xg, None, _t(ism), 0.02, tolerance=1e-12, max_iter=20)
        args = [a if a is not None else np.zeros(0, d) for a, d in
                zip(sets, (H.TRI_DTYPE, H.B1_DTYPE, H.B2_DTYPE, H.B3_DTYPE))]
        xo, _, _ = H.constrain_position(H.clusters(*args), xp, x, ism, 0.02)
        assert np.abs(xg.cpu().numpy().reshape(-1, 3) - xo).max() < 1e-10
    cs = Constraints()
    xg = _t(x)
    cs.position(_t(xp), xg, None, _t(ism), 0.02)
    assert np.array_equal(xg.cpu().numpy(), np.ascontiguousarray(x, np.float64).reshape(-1))
