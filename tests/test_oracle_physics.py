"""CPU oracle: pair physics pinned by the reference's own self-check.

The reference ships no golden vectors for this path; its correctness check is
the finite-difference tester ``run test`` (src/run/run.cu:448-526), which
compares analytic dU/dx and dU/dlambda with central energy differences.  These
tests apply the same check to the FP64 oracle, plus closed-form values of the
pair terms restated independently with numpy/scipy.
"""
import math

import numpy as np
import pytest
from scipy.special import erfc

import oracle
from blade_b200 import systems


@pytest.fixture(scope="module")
def water():
    return systems.water_box()


@pytest.fixture(scope="module")
def msld():
    return systems.msld_water()


def test_cell_list_matches_brute_force(water, msld):
    for s in (water, msld):
        a = oracle.nbdirect(s)
        b = oracle.nbdirect(s, brute=True)
        assert a["pairs"] == b["pairs"] > 0
        assert abs(a["energy"] - b["energy"]) < 1e-9 * max(1.0, abs(a["energy"]))
        np.testing.assert_allclose(a["grad"], b["grad"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(a["lambdaForce"], b["lambdaForce"], rtol=0, atol=1e-9)


def test_pair_count_water216(water):
    # 216 waters, rc 9 A: about 9.2e4 in-cutoff non-excluded pairs
    r = oracle.nbdirect(water)
    assert 80000 < r["pairs"] < 110000


def test_newton_third_law(water):
    g = oracle.nbdirect(water)["grad"]
    assert np.abs(g.sum(0)).max() < 1e-9 * np.abs(g).max() * len(g)


def _fd_x(s, atoms, h=1e-5):
    x = s.xyz.astype(np.float64)
    g = oracle.nbdirect(s, xyz=x)["grad"]
    for a in atoms:
        for d in range(3):
            xp = x.copy(); xp[a, d] += h
            xm = x.copy(); xm[a, d] -= h
            fd = (oracle.nbdirect(s, xyz=xp)["energy"] - oracle.nbdirect(s, xyz=xm)["energy"]) / (2 * h)
            assert abs(fd - g[a, d]) <= 2e-6 * max(1.0, abs(g[a, d])), (a, d, fd, g[a, d])


@pytest.mark.parametrize("elec,vdw", [(e, 0) for e in range(3)])
def test_fd_gradient_all_methods(water, elec, vdw):
    s = systems.water_box()
    s.elecMethod, s.vdwMethod = elec, vdw
    _fd_x(s, [0, 1, 77])


def test_vswitch_force_restates_reference():
    """VSWITCH (vdwMethod 1) keeps the reference's force expression.

    nbdirect.cu:367-368 adds dfsw*(c12/r^6-c6)/r^6 to dE/dr, where the exact
    derivative of its own energy (nbdirect.cu:370) needs an extra factor r.
    The oracle (and the CUDA kernel) reproduce the reference's force, so the
    finite-difference check passes only after restoring that factor.
    """
    s = systems.water_box()
    s.elecMethod, s.vdwMethod = 2, 1
    c12, c6 = 1e5, 5e2
    ron2, roff2 = s.rSwitch ** 2, s.rCut ** 2
    rul3 = (roff2 - ron2) ** 3
    for r in (8.3, 8.7):
        h = 1e-6
        fd = (oracle.pair(r + h, 0, 0, c12, c6, 0, 0, 1, 1, s)[0] -
              oracle.pair(r - h, 0, 0, c12, c6, 0, 0, 1, 1, s)[0]) / (2 * h)
        an = oracle.pair(r, 0, 0, c12, c6, 0, 0, 1, 1, s)[1] * r
        dfsw = (ron2 - r * r) * (roff2 - r * r) * 12 / rul3
        V = (c12 * r ** -6 - c6) * r ** -6
        assert an != pytest.approx(fd, rel=1e-3)
        assert an + dfsw * V * (r - 1) == pytest.approx(fd, rel=1e-7)
    _fd_x_inside_switch = oracle.pair(7.0, 0.3, -0.3, c12, c6, 0, 0, 1, 1, s)
    assert np.isfinite(_fd_x_inside_switch).all()


def test_vshift_force_restates_reference():
    """VSHIFT (vdwMethod 2) keeps the reference's force expression.

    nbdirect.cu:389-390 uses -12*c12*(r^-13 + r^5/rc^18); the derivative of its
    energy (nbdirect.cu:393-394) has -12*c12*(r^-13 - r^5/rc^18).  The oracle
    and the CUDA kernel reproduce the reference; the difference is the
    24*c12*r^5/rc^18 term.
    """
    s = systems.water_box()
    s.elecMethod, s.vdwMethod = 2, 2
    c12, c6 = 1e5, 5e2
    for r in (3.0, 6.0, 8.9):
        h = 1e-6
        fd = (oracle.pair(r + h, 0, 0, c12, c6, 0, 0, 1, 1, s)[0] -
              oracle.pair(r - h, 0, 0, c12, c6, 0, 0, 1, 1, s)[0]) / (2 * h)
        an = oracle.pair(r, 0, 0, c12, c6, 0, 0, 1, 1, s)[1] * r
        assert an + 24 * c12 * r ** 5 / s.rCut ** 18 == pytest.approx(fd, rel=1e-6, abs=1e-12)


def test_fd_gradient_msld_softcore(msld):
    _fd_x(msld, [0, 3, 40, 200])


def test_fd_lambda_msld_softcore(msld):
    lam = msld.lambdas()
    lf = oracle.nbdirect(msld, lam=lam)["lambdaForce"]
    h = 1e-6
    for b in range(1, msld.msld.blockCount):
        lp = lam.copy(); lp[b] += h
        lm = lam.copy(); lm[b] -= h
        fd = (oracle.nbdirect(msld, lam=lp)["energy"] - oracle.nbdirect(msld, lam=lm)["energy"]) / (2 * h)
        assert abs(fd - lf[b]) <= 1e-6 * max(1.0, abs(lf[b])), (b, fd, lf[b])


def test_fd_lambda_without_softcore(msld):
    s = systems.msld_water()
    s.msld.useSoftCore = False
    lam = s.lambdas()
    lf = oracle.nbdirect(s, lam=lam)["lambdaForce"]
    h = 1e-6
    for b in (1, 6, 12):
        lp = lam.copy(); lp[b] += h
        lm = lam.copy(); lm[b] -= h
        fd = (oracle.nbdirect(s, lam=lp)["energy"] - oracle.nbdirect(s, lam=lm)["energy"]) / (2 * h)
        assert abs(fd - lf[b]) <= 1e-6 * max(1.0, abs(lf[b]))


def test_pme_vfswitch_closed_form():
    """E and dE/dr of one pair against an independent numpy restatement."""
    s = systems.water_box()
    rc, rs, beta, k = s.rCut, s.rSwitch, s.betaEwald, 332.0716
    qi, qj, c12, c6 = -0.834, 0.417, 1.2e5, 6.0e2
    for r in (1.7, 3.0, 7.5, 8.5, 8.99):
        E, fr, _, _ = oracle.pair(r, qi, qj, c12, c6, 0, 0, 1.0, 1.0, s)
        ee = k * qi * qj * erfc(beta * r) / r
        de = -k * qi * qj * (erfc(beta * r) / r + 2 * beta / math.sqrt(math.pi) * math.exp(-(beta * r) ** 2)) / r
        rc3, rs3 = rc ** 3, rs ** 3
        if r < rs:
            dv6 = 1 / (rc3 * rs3)
            el = c12 * (r ** -12 - dv6 ** 2) - c6 * (r ** -6 - dv6)
            dl = -12 * c12 * r ** -13 + 6 * c6 * r ** -7
        else:
            k6, k12 = rc3 / (rc3 - rs3), rc3 ** 2 / (rc3 ** 2 - rs3 ** 2)
            el = c12 * k12 * (r ** -6 - rc3 ** -2) ** 2 - c6 * k6 * (r ** -3 - rc3 ** -1) ** 2
            dl = c12 * k12 * 2 * (r ** -6 - rc3 ** -2) * (-6 * r ** -7) - c6 * k6 * 2 * (r ** -3 - rc3 ** -1) * (-3 * r ** -4)
        assert E == pytest.approx(ee + el, rel=1e-12, abs=1e-12)
        assert fr * r == pytest.approx(de + dl, rel=1e-10, abs=1e-10)


@pytest.mark.parametrize("elec,vdw", [(0, 0), (0, 1), (2, 2), (2, 0)])
def test_switched_energy_vanishes_at_cutoff(elec, vdw):
    s = systems.water_box()
    s.elecMethod, s.vdwMethod = elec, vdw
    E, fr, _, _ = oracle.pair(s.rCut * (1 - 1e-9), 0.5, -0.5, 1e5, 5e2, 0, 0, 1, 1, s)
    assert abs(E) < 1e-6
    if vdw != 2 and elec != 2:
        assert abs(fr) < 1e-6


def test_msld_scaling_rules():
    """Scale and dU/dlambda routing of nbdirect.cu:244-256,400-415."""
    s = systems.msld_water()
    s.msld.useSoftCore = False
    p = oracle.params(s)
    r, qi, qj, c12, c6 = 5.0, 0.3, -0.4, 1e5, 5e2
    E0, _, _, _ = oracle.pair(r, qi, qj, c12, c6, 0, 0, 1, 1, p)
    bA, bB, bC = (1 << 16) | 1, (1 << 16) | 2, (2 << 16) | 5
    # environment-environment (lambda of the environment block is 1): unscaled
    p.calcAlch = 1
    assert oracle.pair(r, qi, qj, c12, c6, 0, 0, 1.0, 1.0, p)[0] == pytest.approx(E0)
    # env - perturbed: scaled by lambda_j, force routed to j only
    E, _, fli, flj = oracle.pair(r, qi, qj, c12, c6, 0, bA, 1.0, 0.25, p)
    assert E == pytest.approx(0.25 * E0) and flj == pytest.approx(E0) and fli == pytest.approx(0.25 * E0)
    # same block: scaled by lambda_i once
    E, _, fli, flj = oracle.pair(r, qi, qj, c12, c6, bA, bA, 0.4, 0.4, p)
    assert E == pytest.approx(0.4 * E0) and fli == pytest.approx(E0) and flj == 0
    # same site, different block: no interaction
    E, fr, fli, flj = oracle.pair(r, qi, qj, c12, c6, bA, bB, 0.4, 0.5, p)
    assert E == 0 and fr == 0 and fli == 0 and flj == 0
    # different sites: lambda_i * lambda_j
    E, _, fli, flj = oracle.pair(r, qi, qj, c12, c6, bA, bC, 0.4, 0.5, p)
    assert E == pytest.approx(0.2 * E0) and fli == pytest.approx(0.5 * E0) and flj == pytest.approx(0.4 * E0)


def test_softcore_caps_close_contact():
    s = systems.msld_water()
    p = oracle.params(s)
    b = (1 << 16) | 1
    E_hard = oracle.pair(0.3, 0.5, -0.5, 1e5, 5e2, 0, 0, 1, 1, p)[0]
    E_soft = oracle.pair(0.3, 0.5, -0.5, 1e5, 5e2, 0, b, 1, 0.2, p)[0]
    assert abs(E_soft) < 1e3 < abs(E_hard)
