"""nb14 / nbex pair lists on the GPU (bnb_compute_nb14 / bnb_compute_nbex)
against the FP64 oracle: every method combination, MSLD scaling with and
without the 1-4 soft core, two replicas on one handle, and repeated calls."""
import numpy as np
import pytest

import oracle
from blade_b200 import systems
from blade_b200.nbdirect import NbDirect

pytestmark = pytest.mark.gpu

FORCE_TOL = 2e-5      # relative RMS of dU/dx vs FP64 (FP32 pair math, fixed-point sums)
ENERGY_TOL = 1e-5
DUDL_TOL = 5e-5


def _rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


@pytest.fixture(scope="module")
def chain():
    return systems.with_pair_lists(systems.chain_in_water(seed=5, box=30.0, n_chain=250, n_wat=780, name="c"),
                                   e14fac=0.5)


def _check(s, which, soft=False, nb=None):
    own = nb is None
    nb = nb or NbDirect(s)
    nb.set_pairs(soft14=soft)
    f, l, e = nb.evaluate_pairs(which)
    o = oracle.pair_lists(s, which=which, soft14=soft)
    assert _rel(f.cpu().numpy(), o["grad"]) < FORCE_TOL
    assert float(e.cpu()[0]) == pytest.approx(o["energy"], rel=ENERGY_TOL)
    if s.msld:
        assert _rel(l.cpu().numpy()[1:], o["lambdaForce"][1:]) < DUDL_TOL
    if own:
        nb.close()


@pytest.mark.parametrize("elec", [0, 1, 2])
@pytest.mark.parametrize("vdw", [0, 1, 2])
def test_nb14_matches_oracle(cuda, chain, elec, vdw):
    chain.elecMethod, chain.vdwMethod = elec, vdw
    _check(chain, "nb14")


def test_nbex_matches_oracle(cuda, chain):
    chain.elecMethod, chain.vdwMethod = 1, 0
    _check(chain, "nbex")


@pytest.mark.parametrize("soft", [False, True])
def test_msld_pairs(cuda, soft):
    s = systems.with_pair_lists(systems.msld_water())
    _check(s, "nb14", soft=soft)
    _check(s, "nbex")


def test_two_replicas_and_repeat(cuda):
    reps = [systems.with_pair_lists(systems.msld_water(3 + k)) for k in range(2)]
    nb = NbDirect(reps)
    nb.set_pairs(soft14=True)
    for _ in range(2):                       # accumulators are left at zero between calls
        f, l, e = nb.evaluate_pairs("nb14")
        for r, s in enumerate(reps):
            o = oracle.pair_lists(s, which="nb14", soft14=True)
            a0, a1 = nb.starts[r], nb.starts[r + 1]
            assert _rel(f.cpu().numpy()[a0:a1], o["grad"]) < FORCE_TOL
            assert float(e.cpu()[r]) == pytest.approx(o["energy"], rel=ENERGY_TOL)
            l0, l1 = nb.lam_starts[r], nb.lam_starts[r + 1]
            assert _rel(l.cpu().numpy()[l0 + 1:l1], o["lambdaForce"][1:]) < DUDL_TOL
    nb.close()


@pytest.mark.parametrize("name", ["pairs_nb14_e1v0", "pairs_nb14_e0v1", "pairs_nb14_e2v2", "pairs_nbex",
                                  "pairs_msld_nb14_soft", "pairs_msld_nb14_hard", "pairs_msld_nbex"])
def test_gpu_matches_reference_pairs(cuda, name):
    import os
    from test_golden_pairs import DUDL_TOL as DT, ENERGY_TOL as ET, FORCE_TOL as FT, case, rel_rms
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    s, which, soft = case(name)
    s.elecMethod, s.vdwMethod = int(z["elecMethod"]), int(z["vdwMethod"])
    nb = NbDirect(s)
    nb.set_pairs(soft14=soft)
    f, l, e = nb.evaluate_pairs(which)
    n = int(z["n_forces"])
    assert rel_rms(f.cpu().numpy()[:n], z["grad"]) < FT
    assert float(e.cpu()[0]) == pytest.approx(float(z["energy"]), rel=ET)
    if s.msld:
        assert rel_rms(l.cpu().numpy()[1:], z["lambdaForce"][1:]) < DT
    nb.close()
