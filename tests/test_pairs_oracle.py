"""FP64 oracle of the nb14 / nbex pair lists (src/bonded/pair.cu): gradients
against central finite differences for every method combination, dU/dlambda
against finite differences in lambda, and Newton's third law."""
import numpy as np
import pytest

import oracle
from blade_b200 import systems


@pytest.fixture(scope="module")
def chain():
    return systems.with_pair_lists(systems.chain_in_water(seed=5, box=30.0, n_chain=120, n_wat=300, name="c"),
                                   e14fac=0.5)


def _fd(s, which, x, atom, k, h=1e-5, **kw):
    xp, xm = x.copy(), x.copy()
    xp[atom, k] += h
    xm[atom, k] -= h
    return (oracle.pair_lists(s, xyz=xp, which=which, **kw)["energy"]
            - oracle.pair_lists(s, xyz=xm, which=which, **kw)["energy"]) / (2 * h)


def test_lists(chain):
    assert len(chain.nb14) == 117                 # (i, i+3) along a 120-atom chain
    ex = set(map(tuple, chain.excl.tolist()))
    assert all((int(i), int(j)) in ex for i, j in chain.nb14["idx"])
    assert not set(map(tuple, chain.nbex["idx"].tolist())) & set(map(tuple, chain.nb14["idx"].tolist()))


@pytest.mark.parametrize("elec", [0, 1, 2])
@pytest.mark.parametrize("vdw", [0, 1, 2])
def test_nb14_gradient(chain, elec, vdw):
    s = chain
    s.elecMethod, s.vdwMethod = elec, vdw
    x = s.xyz.astype(np.float64)
    g = oracle.pair_lists(s, xyz=x, which="nb14")["grad"]
    rng = np.random.default_rng(elec * 3 + vdw)
    for _ in range(6):
        a = int(s.nb14[rng.integers(len(s.nb14))]["idx"][rng.integers(2)])
        k = int(rng.integers(3))
        fd = _fd(s, "nb14", x, a, k)
        assert fd == pytest.approx(g[a, k], rel=1e-6, abs=1e-6)
    np.testing.assert_allclose(g.sum(0), 0, atol=1e-8)


def test_nbex_gradient(chain):
    s = chain
    s.elecMethod, s.vdwMethod = 1, 0
    x = s.xyz.astype(np.float64)
    g = oracle.pair_lists(s, xyz=x, which="nbex")["grad"]
    for a in (0, 5, 130, 131):
        for k in range(3):
            assert _fd(s, "nbex", x, a, k) == pytest.approx(g[a, k], rel=1e-6, abs=1e-6)


@pytest.mark.parametrize("soft", [False, True])
def test_msld_dudlambda(soft):
    s = systems.with_pair_lists(systems.msld_water())
    lam = s.lambdas()
    o = oracle.pair_lists(s, lam=lam, which="nb14", soft14=soft)
    h = 1e-6
    for b in (1, 5, 9):
        lp, lm = lam.copy(), lam.copy()
        lp[b] += h
        lm[b] -= h
        fd = (oracle.pair_lists(s, lam=lp, which="nb14", soft14=soft)["energy"]
              - oracle.pair_lists(s, lam=lm, which="nb14", soft14=soft)["energy"]) / (2 * h)
        assert fd == pytest.approx(o["lambdaForce"][b], rel=1e-5, abs=1e-6)
    oe = oracle.pair_lists(s, lam=lam, which="nbex")
    for b in (2, 6):
        lp, lm = lam.copy(), lam.copy()
        lp[b] += h
        lm[b] -= h
        fd = (oracle.pair_lists(s, lam=lp, which="nbex")["energy"]
              - oracle.pair_lists(s, lam=lm, which="nbex")["energy"]) / (2 * h)
        assert fd == pytest.approx(oe["lambdaForce"][b], rel=1e-5, abs=1e-6)
