"""The FP64 PME restatement against golden vectors made by the reference's
own getforce_ewald / getforce_ewaldself (src/nbrecip/nbrecip.cu, FP32 with
cuFFT, built unmodified; tests/golden/make_golden.py --pme-only): orders 4,
6 and 8 on the water box, MSLD lambda scaling, and a chain-in-water box."""
import glob
import os

import numpy as np
import pytest

from blade_b200 import systems
from oracle import pme_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "pme_*.npz")))
FORCE_TOL, ENERGY_TOL, DUDL_TOL = 1e-5, 5e-6, 1e-5   # the reference computes in FP32
K_ELECTRIC = 332.0716


def case(name):
    if name.startswith("pme_msld"):
        return systems.msld_water()
    if name.startswith("pme_chain"):
        return systems.chain_in_water(seed=5, box=30.0, n_chain=250, n_wat=780, name="chain_water_small")
    return systems.water_box()


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def test_files_present():
    assert len(FILES) == 5


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_oracle_matches_reference_pme(path):
    z = np.load(path)
    s = case(os.path.basename(path)[:-4])
    assert np.array_equal(s.xyz, z["xyz"]), "generator drifted from the fixture"
    K = [int(k) for k in z["K"]]
    assert K == [pme_oracle.grid_size(L, 1.0) for L in s.box]
    lam = s.lambdas() if s.msld else None
    sb = s.nbonds["siteBlock"]
    E, g, lf, _ = pme_oracle.pme_recip(s.xyz, s.nbonds["q"], s.box, K, int(z["order"]), s.betaEwald, K_ELECTRIC,
                                       sb, lam)
    assert rel_rms(g, z["grad"]) < FORCE_TOL
    assert E == pytest.approx(float(z["energy"]), rel=ENERGY_TOL)
    Es, ls = pme_oracle.ewald_self(s.nbonds["q"], s.betaEwald, K_ELECTRIC, sb, lam)
    assert Es == pytest.approx(float(z["self_energy"]), rel=1e-6)
    if lam is not None:
        assert rel_rms(lf[1:], z["lambdaForce"][1:]) < DUDL_TOL
        assert rel_rms(ls[1:], z["self_lambdaForce"][1:]) < 1e-6
