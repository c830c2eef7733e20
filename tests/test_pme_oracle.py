"""The FP64 PME restatement (oracle/pme_oracle.py) on its own: the grid rule
of Potential::initialize, B-spline identities, convergence to the plain Ewald
reciprocal sum, and finite-difference checks of dU/dx and dU/dlambda."""
import numpy as np
import pytest

from blade_b200 import systems
from oracle import pme_oracle as P

K_ELECTRIC = 332.0716


def test_grid_rule():
    # L / spacing -> smallest of j*{32,27,24,20,18} above it (potential.cxx:1204-1218)
    cases = {62.23: 64, 18.856: 20, 40.0: 48, 100.0: 108, 12.0: 18, 30.0: 32, 25.14: 27, 17.9: 18, 33.0: 36}
    for L, K in cases.items():
        assert P.grid_size(L, 1.0) == K, L
    assert P.grid_size(62.23, 0.5) == 128


def test_bspline_identities():
    f = np.linspace(0.0, 0.999, 17)
    for n in (4, 6, 8):
        w, d = P.weights(f, n)
        assert np.allclose(w.sum(-1), 1.0, atol=1e-14)      # partition of unity
        assert np.allclose(d.sum(-1), 0.0, atol=1e-14)
        assert np.all(w >= 0)
        M = P.bspline_int(n)
        assert M.sum() == pytest.approx(1.0)
        # weights at f = 0 are M_n at the integers n-1 .. 0
        w0, _ = P.weights(np.zeros(1), n)
        assert np.allclose(w0[0], M[n - 1::-1][:n])
        h = 1e-6
        fi = f[1:]                                           # interior points: f - h stays >= 0
        wp, _ = P.weights(fi + h, n)
        wm, _ = P.weights(fi - h, n)
        assert np.allclose((wp - wm) / (2 * h), d[1:], atol=1e-6)


def test_converges_to_ewald_sum():
    s = systems.water_box()
    q = s.nbonds["q"].astype(np.float64)
    E0, g0 = P.ewald_recip_exact(s.xyz, q, s.box, 0.34, K_ELECTRIC, kmax=12)
    E, g, _, _ = P.pme_recip(s.xyz, q, s.box, [48, 48, 48], 8, 0.34, K_ELECTRIC)
    assert E == pytest.approx(E0, rel=1e-8)
    assert np.sqrt(((g - g0) ** 2).sum() / (g0 ** 2).sum()) < 1e-8
    # the reference's default (1 A grid, order 6) is within 1e-4
    E6, g6, _, _ = P.pme_recip(s.xyz, q, s.box, [20, 20, 20], 6, 0.34, K_ELECTRIC)
    assert E6 == pytest.approx(E0, rel=2e-4)


def test_finite_differences():
    s = systems.msld_water()
    q = s.nbonds["q"].astype(np.float64)
    sb = s.nbonds["siteBlock"]
    lam = s.lambdas().astype(np.float64)
    K = [P.grid_size(L, 1.0) for L in s.box]
    E, g, lf, _ = P.pme_recip(s.xyz, q, s.box, K, 6, s.betaEwald, K_ELECTRIC, sb, lam)
    x0 = s.xyz.astype(np.float64)
    h = 1e-5
    pert = np.nonzero(sb & 0xFFFF)[0]
    for i in (0, 7, int(pert[0]), int(pert[-1])):
        for d in range(3):
            xp = x0.copy(); xp[i, d] += h
            xm = x0.copy(); xm[i, d] -= h
            fd = (P.pme_recip(xp, q, s.box, K, 6, s.betaEwald, K_ELECTRIC, sb, lam)[0]
                  - P.pme_recip(xm, q, s.box, K, 6, s.betaEwald, K_ELECTRIC, sb, lam)[0]) / (2 * h)
            assert fd == pytest.approx(g[i, d], rel=1e-5, abs=1e-6)
    for b in range(1, len(lam)):
        lp = lam.copy(); lp[b] += 1e-6
        lm = lam.copy(); lm[b] -= 1e-6
        fd = (P.pme_recip(x0, q, s.box, K, 6, s.betaEwald, K_ELECTRIC, sb, lp)[0]
              - P.pme_recip(x0, q, s.box, K, 6, s.betaEwald, K_ELECTRIC, sb, lm)[0]) / 2e-6
        assert fd == pytest.approx(lf[b], rel=1e-5, abs=1e-5)
    Es, ls = P.ewald_self(q, s.betaEwald, K_ELECTRIC, sb, lam)
    for b in range(1, len(lam)):
        lp = lam.copy(); lp[b] += 1e-6
        lm = lam.copy(); lm[b] -= 1e-6
        fd = (P.ewald_self(q, s.betaEwald, K_ELECTRIC, sb, lp)[0] - P.ewald_self(q, s.betaEwald, K_ELECTRIC, sb, lm)[0]) / 2e-6
        assert fd == pytest.approx(ls[b], rel=1e-6, abs=1e-6)


def test_translation_invariance():
    """A shift of every atom by whole grid cells leaves energy and forces
    unchanged (the grid convention is a translation of the reference's)."""
    s = systems.water_box()
    q = s.nbonds["q"].astype(np.float64)
    K = [20, 20, 20]
    E, g, _, _ = P.pme_recip(s.xyz, q, s.box, K, 6, 0.34, K_ELECTRIC)
    shift = np.float64(s.box[0]) / 20 * np.array([3, -1, 7])
    E2, g2, _, _ = P.pme_recip(s.xyz.astype(np.float64) + shift, q, s.box, K, 6, 0.34, K_ELECTRIC)
    assert E2 == pytest.approx(E, rel=1e-10)
    assert np.allclose(g2, g, atol=1e-8)


def test_total_electrostatics_is_beta_invariant():
    """Direct space (erfc, cutoff) + nbex exclusion corrections + PME
    reciprocal + self term is the Ewald sum, whose value does not depend on
    the splitting parameter beta: beta 0.34 and 0.40 agree to the direct-space
    truncation erfc(beta rCut) (1.2e-5 at beta 0.34, rCut 9 A) of the
    components' scale."""
    import dataclasses as dc
    import oracle
    base = systems.with_pair_lists(systems.water_box())
    q = base.nbonds["q"].astype(np.float64)
    totals, scale = [], 0.0
    for beta in (0.34, 0.40):
        s = dc.replace(base, betaEwald=beta)
        parts = (oracle.nbdirect(s)["energy"], oracle.pair_lists(s, which="nbex")["energy"],
                 P.pme_recip(s.xyz, q, s.box, [40, 40, 40], 8, beta, K_ELECTRIC)[0],
                 P.ewald_self(q, beta, K_ELECTRIC)[0])
        totals.append(sum(parts))
        scale = max(scale, max(abs(p) for p in parts))
    assert abs(totals[0] - totals[1]) < 2e-5 * scale


def test_triclinic_converges_to_ewald_sum():
    """In a triclinic cell (fractional coordinates H^-1 x, k = H^-T m) the
    restatement converges to the plain Ewald sum over the cell's k vectors."""
    s = systems.water_box_tric()
    q = s.nbonds["q"].astype(np.float64)
    box6 = s.box6()
    E0, g0 = P.ewald_recip_exact(s.xyz, q, box6, 0.34, K_ELECTRIC, kmax=14)
    E, g, _, _ = P.pme_recip(s.xyz, q, box6, [64, 48, 64], 8, 0.34, K_ELECTRIC)
    assert E == pytest.approx(E0, rel=1e-7)
    assert np.sqrt(((g - g0) ** 2).sum() / (g0 ** 2).sum()) < 1e-6


def test_triclinic_orthorhombic_cell_equals_edge_lengths():
    s = systems.water_box()
    q = s.nbonds["q"].astype(np.float64)
    K = [20, 20, 20]
    E, g, _, _ = P.pme_recip(s.xyz, q, s.box, K, 6, 0.34, K_ELECTRIC)
    box6 = np.concatenate([np.asarray(s.box, np.float64), np.zeros(3)])
    E6, g6, _, _ = P.pme_recip(s.xyz, q, box6, K, 6, 0.34, K_ELECTRIC)
    assert E6 == E and np.array_equal(g6, g)
    assert np.allclose(P.edge_lengths(box6), s.box)


def test_triclinic_finite_differences_and_lattice_moves():
    s = systems.water_box_tric()
    q = s.nbonds["q"].astype(np.float64)
    box6 = s.box6()
    K = [P.grid_size(L, 1.0) for L in P.edge_lengths(box6)]
    x0 = s.xyz.astype(np.float64)
    E, g, _, _ = P.pme_recip(x0, q, box6, K, 6, s.betaEwald, K_ELECTRIC)
    h = 1e-5
    for i in (0, 5, 400):
        for d in range(3):
            xp = x0.copy(); xp[i, d] += h
            xm = x0.copy(); xm[i, d] -= h
            fd = (P.pme_recip(xp, q, box6, K, 6, s.betaEwald, K_ELECTRIC)[0]
                  - P.pme_recip(xm, q, box6, K, 6, s.betaEwald, K_ELECTRIC)[0]) / (2 * h)
            assert fd == pytest.approx(g[i, d], rel=1e-5, abs=1e-6)
    H, _ = P.cell(box6)
    moved = x0 + np.random.default_rng(2).integers(-2, 3, (len(x0), 3)) @ H.T
    E2, g2, _, _ = P.pme_recip(moved, q, box6, K, 6, s.betaEwald, K_ELECTRIC)
    assert E2 == pytest.approx(E, rel=1e-10)
    assert np.allclose(g2, g, atol=1e-7)
