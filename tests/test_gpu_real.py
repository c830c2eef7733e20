"""libbnb on the reference's own CHARMM fixtures (test/water216,
test/newDHFR; see tests/test_golden_real.py): direct space through the block
list, the nb14 / nbex pair lists and PME against the reference's own CUDA
outputs and the FP64 oracle, and the pair count against the oracle's.  DHFR
has 35 LJ types, so this is the per-pair-table pair kernel at protein scale."""
import numpy as np
import pytest
import torch

import oracle
from blade_b200.nbdirect import NbDirect
from oracle import pme_oracle

from test_golden_real import NAMES, energy_ok, load, rel_rms

pytestmark = pytest.mark.gpu
ORACLE_FORCE_TOL = 1e-5    # relative RMS of dU/dx vs FP64
REF_FORCE_TOL = 1e-5       # vs the reference's FP32 build
ENERGY_TOL = 1e-5          # per max(|E|, N)
PME_FORCE_TOL = 5e-5       # FP32 B-splines and FFT against the reference's FP32 grid
K_ELECTRIC = 332.0716


@pytest.mark.parametrize("name", NAMES)
def test_direct_space(cuda, name):
    s, z = load(name)
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    nb.set_counting(True)
    f, _, e = nb.evaluate(pos)
    torch.cuda.synchronize()
    assert nb.status() == 0
    g = f.cpu().numpy()
    o = oracle.nbdirect(s)
    assert nb.pair_count() == o["pairs"]
    assert rel_rms(g, o["grad"]) <= ORACLE_FORCE_TOL
    assert rel_rms(g, z["grad"].astype(np.float64)) <= REF_FORCE_TOL
    assert energy_ok(float(e[0]), o["energy"], s.N, ENERGY_TOL)
    assert energy_ok(float(e[0]), float(z["energy"]), s.N, ENERGY_TOL)
    nb.close()


@pytest.mark.parametrize("name", NAMES)
def test_pair_lists(cuda, name):
    s, z = load(name)
    nb = NbDirect(s)
    nb.set_pairs()
    for which, key in (("nb14", "14"), ("nbex", "ex")):
        if which == "nb14" and not len(s.nb14):
            continue
        f, _, e = nb.evaluate_pairs(which)
        torch.cuda.synchronize()
        g = f.cpu().numpy()
        o = oracle.pair_lists(s, which=which)
        assert rel_rms(g, o["grad"]) <= ORACLE_FORCE_TOL, which
        assert rel_rms(g, z["grad" + key].astype(np.float64)) <= REF_FORCE_TOL, which
        assert energy_ok(float(e[0]), float(z["energy" + key]), s.N, ENERGY_TOL), which
    nb.close()


@pytest.mark.parametrize("name", NAMES)
def test_pme(cuda, name):
    s, z = load(name)
    K = [int(k) for k in z["K"]]
    nb = NbDirect(s)
    nb.set_pme(order=int(z["order"]), grid=K)
    assert list(nb.pme_grid()) == K
    f, _, e = nb.evaluate_pme()
    _, es = nb.evaluate_ewald_self()
    torch.cuda.synchronize()
    g = f.cpu().numpy()
    E, go, _, _ = pme_oracle.pme_recip(s.xyz, s.nbonds["q"], s.box, K, int(z["order"]), s.betaEwald, K_ELECTRIC)
    assert rel_rms(g, go) <= 2e-5
    assert rel_rms(g, z["gradpme"].astype(np.float64)) <= PME_FORCE_TOL
    assert energy_ok(float(e[0]), E, s.N, ENERGY_TOL)
    assert float(es[0]) == pytest.approx(float(z["energyself"]), rel=1e-6)
    nb.close()
