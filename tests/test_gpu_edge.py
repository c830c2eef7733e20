"""GPU edge cases: capacity overflow and regrowth, asynchronous overflow
reporting, non-finite input, tiny and uneven systems, MSLD lambda kernels."""
import dataclasses

import numpy as np
import pytest
import torch

import oracle
from blade_b200 import msld as gmsld
from blade_b200 import systems, _lib
from blade_b200.nbdirect import NbDirect

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def test_overflow_regrows_in_sync_rebuild(cuda):
    """Undersized tile/mask/work capacities grow like cull.cu:337-375."""
    s = systems.water_box()
    nb = NbDirect(s)
    nb.reserve(tiles=16, masks=2, work=4)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    assert nb.status() & 15 == 0
    f, _, e = nb.evaluate(pos)
    o = oracle.nbdirect(s)
    assert rel_rms(f.cpu().numpy(), o["grad"]) <= 1e-5
    nb.close()


def test_async_overflow_is_reported_and_skipped(cuda):
    s = systems.water_box()
    nb = NbDirect(s)
    nb.reserve(tiles=16, masks=2, work=4)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True, asynchronous=True)
    st = nb.status()
    assert st & _lib.STATUS_TILE_OVERFLOW
    f, _, e = nb.evaluate(pos)           # pair kernel does no work on an invalid list
    assert float(f.abs().sum()) == 0.0
    nb.update_domdec(pos, True)          # a synchronous rebuild recovers
    assert nb.status() & 15 == 0
    f, _, _ = nb.evaluate(pos)
    assert rel_rms(f.cpu().numpy(), oracle.nbdirect(s)["grad"]) <= 1e-5
    nb.close()


def test_nonfinite_coordinates_flagged(cuda):
    s = systems.water_box()
    s.xyz = s.xyz.copy()
    s.xyz[5, 1] = np.nan
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    nb.evaluate(pos)
    assert nb.status() & _lib.STATUS_NONFINITE
    nb.close()


def test_small_and_sparse_systems(cuda):
    # a handful of atoms in a big box: blocks with 1-3 atoms, many empty columns
    rng = np.random.default_rng(3)
    s = systems.water_box()
    s.xyz = (rng.uniform(0, 30, (9, 3))).astype(np.float32)
    s.box = np.float32([30, 30, 30])
    s.nbonds = s.nbonds[:9].copy()
    s.excl = s.excl[(s.excl < 9).all(1)]
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    nb.set_counting(True)
    f, _, e = nb.evaluate(pos)
    o = oracle.nbdirect(s)
    assert nb.pair_count() == o["pairs"]
    assert rel_rms(f.cpu().numpy(), o["grad"]) <= 1e-5
    nb.close()


def test_atoms_on_box_faces(cuda):
    s = systems.water_box()
    s.xyz = s.xyz.copy()
    L = float(s.box[0])
    s.xyz[0] = [0.0, 0.0, 0.0]
    s.xyz[3] = [L, L * 0.5, np.nextafter(np.float32(L), np.float32(0))]
    s.xyz[6] = [-0.0, L, 1e-7]
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    g = nb.get_list()
    o = oracle.build_list(s)
    for k in ("wrap", "sortedAtom", "cand", "masks"):
        assert np.array_equal(g[k], o[k]), k
    nb.close()


def test_list_reuse_between_rebuilds(cuda):
    """Positions move between rebuilds; the pad keeps every pair (Domdec freqDomdec)."""
    s = systems.water_box()
    rng = np.random.default_rng(9)
    nb = NbDirect(s)
    nb.update_domdec(nb.positions_tensor(), True)
    x = s.xyz.copy()
    for _ in range(5):
        x = (x + rng.normal(0, 0.08, x.shape)).astype(np.float32)
        pos = nb.positions_tensor([x])
        nb.set_counting(True)
        f, _, _ = nb.evaluate(pos)
        o = oracle.nbdirect(s, xyz=x)
        assert nb.pair_count() == o["pairs"]
        assert rel_rms(f.cpu().numpy(), o["grad"]) <= 1e-5
    nb.close()


def test_msld_lambda_kernels(cuda):
    bound = np.array([0, 1, 4, 8, 11], np.int32)
    site = np.array([0, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3], np.int32)
    rng = np.random.default_rng(2)
    th = rng.uniform(-2, 2, 11)
    th[0] = 1.0
    fixed = np.zeros(11, np.uint8)          # bool layout of Msld::blockFixed_d
    fixed[0] = 1
    dev = lambda a: torch.from_numpy(a).cuda()
    lam = torch.zeros(11, dtype=torch.float64, device="cuda")
    lamf = torch.zeros(11, dtype=torch.float32, device="cuda")
    gmsld.lambda_from_theta(dev(bound), 5.5, dev(th), lam, lamf, dev(fixed))
    ol = oracle.lambda_from_theta(bound, 5.5, th, fixed.astype(np.int32))
    np.testing.assert_allclose(lam.cpu().numpy(), ol, rtol=1e-13, atol=1e-15)
    F = rng.normal(size=11)
    tf = torch.zeros(11, dtype=torch.float64, device="cuda")
    gmsld.theta_force(dev(site), dev(bound), 5.5, lam, dev(th), dev(F), tf, dev(fixed))
    np.testing.assert_allclose(tf.cpu().numpy(),
                               oracle.theta_force(site, bound, 5.5, ol, th, F, fixed.astype(np.int32)),
                               rtol=1e-12, atol=1e-12)
    # FP32-buffer form used with the reference's State buffers
    tf32 = torch.zeros(11, dtype=torch.float32, device="cuda")
    gmsld.theta_force_f32(dev(site), dev(bound), 5.5, lamf, lam.float().new_tensor(th.astype(np.float32)),
                          dev(F.astype(np.float32)), tf32, dev(fixed))
    np.testing.assert_allclose(tf32.cpu().numpy(), tf.cpu().numpy(), rtol=2e-5, atol=2e-5)
    vb = np.zeros(4, gmsld.VARBIAS_DTYPE)
    vb[0] = (1, 2, 6, 0.0, 2.0, 0)
    vb[1] = (1, 3, 8, 0.017, -1.5, 0)
    vb[2] = (4, 5, 10, -5.56, 0.7, 0)
    vb[3] = (5, 9, 6, 0.0, 3.0, 0)
    fb = rng.normal(size=11)
    lf = torch.zeros(11, dtype=torch.float64, device="cuda")
    en = torch.zeros(1, dtype=torch.float64, device="cuda")
    vbd = torch.from_numpy(vb.view(np.uint8).copy()).cuda()
    gmsld.bias(lam, dev(fb), vbd, lf, en)
    olf, oe = oracle.bias(ol, fb, vb)
    np.testing.assert_allclose(lf.cpu().numpy(), olf, rtol=1e-5, atol=1e-6)
    assert float(en[0]) == pytest.approx(oe, rel=1e-6)


def test_output_modes(cuda):
    """BNB_OUT_SET overwrites force / lambdaForce / energy; BNB_OUT_ADD64 adds
    into force64 / lambdaForce64 / energy64; the default adds and overwrites."""
    from blade_b200 import _lib
    s = systems.msld_water()
    nb = NbDirect(s)
    pos, lam = nb.positions_tensor(), nb.lambdas_tensor()
    nb.update_domdec(pos, True)
    f64, l64, e64 = nb.evaluate(pos, lam)
    N3, L = 3 * s.N, nb.L
    f = torch.full((N3,), 7.0, device="cuda")
    lf = torch.full((L,), -3.0, device="cuda")
    e = torch.full((1,), 11.0, dtype=torch.float64, device="cuda")
    nb.getforce_nbdirect(pos, lam, True, force=f, lambda_force=lf, energy=e, mode=_lib.BNB_OUT_SET)
    torch.cuda.synchronize()
    assert torch.allclose(f.double(), f64.reshape(-1), rtol=1e-6, atol=1e-5)
    assert torch.allclose(lf.double(), l64, rtol=1e-6, atol=1e-5)
    assert float(e[0]) == float(e64[0])
    g = torch.full((N3,), 2.5, dtype=torch.float64, device="cuda")
    gl = torch.full((L,), 1.5, dtype=torch.float64, device="cuda")
    ge = torch.full((1,), -4.0, dtype=torch.float64, device="cuda")
    nb.getforce_nbdirect(pos, lam, True, force64=g, lambda_force64=gl, energy64=ge, mode=_lib.BNB_OUT_ADD64)
    torch.cuda.synchronize()
    assert torch.equal(g, 2.5 + f64.reshape(-1))
    assert torch.equal(gl, 1.5 + l64)
    assert float(ge[0]) == -4.0 + float(e64[0])
    with pytest.raises(_lib.BnbError):
        nb.getforce_nbdirect(pos, lam, True, force64=g, mode=8)
    nb.close()


def test_pair_erfc_path_against_fp64(cuda):
    """One charge pair at distances across [0.7 A, rCut): the device path
    erfc(beta r) = ex2(-beta^2 r^2 log2 e) P6(rcp(1 + p beta r)) with rsqrt,
    in the PME real-space energy and force, against FP64 erfc."""
    from math import erfc, exp, pi, sqrt
    s = systems.water_box()
    nb0 = np.zeros(2, systems.NBOND_DTYPE)
    nb0["q"] = (0.83, -0.61)
    vdw = np.zeros((1, 1, 2), np.float32)            # no LJ: the Coulomb term alone
    k, beta, rc = 332.0716, 0.32, 12.0
    worst_e = worst_f = 0.0
    for r in np.concatenate([np.linspace(0.7, 11.9, 57), [11.99]]):
        xyz = np.array([[20.0, 20.0, 20.0], [20.0 + r * 0.6, 20.0 + r * 0.8, 20.0]], np.float32)
        t = dataclasses.replace(s, xyz=xyz, box=np.float32([40.0, 40.0, 40.0]), nbonds=nb0, vdw=vdw,
                                excl=np.zeros((0, 2), np.int32), rCut=rc, rSwitch=10.0, betaEwald=beta,
                                name="pair")
        nb = NbDirect(t)
        pos = nb.positions_tensor()
        nb.update_domdec(pos, True)
        f, _, e = nb.evaluate(pos)
        torch.cuda.synchronize()
        d = xyz[0].astype(np.float64) - xyz[1].astype(np.float64)
        rr = float(np.linalg.norm(d))
        qq = k * float(np.float32(0.83)) * float(np.float32(-0.61))
        E = qq * erfc(beta * rr) / rr
        dEdr = -qq * (erfc(beta * rr) / rr + 2 * beta / sqrt(pi) * exp(-(beta * rr) ** 2)) / rr
        g0 = dEdr * d / rr                           # dU/dx of atom 0
        # relative error, with the 2^-32 quantum of the fixed-point sums as floor
        worst_e = max(worst_e, abs(float(e[0]) - E) / (abs(E) + 1e-3))
        worst_f = max(worst_f, float(np.abs(f.cpu().numpy()[0] - g0).max()) / (float(np.abs(g0).max()) + 1e-3))
        nb.close()
    assert worst_e <= 2e-6, worst_e
    assert worst_f <= 2e-6, worst_f
