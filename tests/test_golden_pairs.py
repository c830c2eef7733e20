"""The FP64 oracle of the nb14 / nbex pair lists against golden vectors made
by the reference's own getforce_nb14 / getforce_nbex (src/bonded/pair.cu,
FP32, built unmodified; tests/golden/make_golden.py --pairs-only)."""
import glob
import os

import numpy as np
import pytest

import oracle
from blade_b200 import systems

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "pairs_*.npz")))
FORCE_TOL, ENERGY_TOL, DUDL_TOL = 2e-5, 2e-5, 5e-5


def case(name):
    base = systems.chain_in_water(seed=5, box=30.0, n_chain=250, n_wat=780, name="chain_water_small")
    if name.startswith("pairs_msld"):
        s = systems.with_pair_lists(systems.msld_water())
    else:
        s = systems.with_pair_lists(base, e14fac=0.5)
    which = "nbex" if name.endswith("nbex") else "nb14"
    return s, which, name.endswith("_soft")


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def test_files_present():
    assert len(FILES) == 7


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_oracle_matches_reference_pairs(path):
    z = np.load(path)
    name = os.path.basename(path)[:-4]
    s, which, soft = case(name)
    s.elecMethod, s.vdwMethod = int(z["elecMethod"]), int(z["vdwMethod"])
    assert np.array_equal(s.xyz, z["xyz"]), "generator drifted from the fixture"
    o = oracle.pair_lists(s, which=which, soft14=soft)
    n = int(z["n_forces"])
    assert rel_rms(o["grad"][:n], z["grad"]) < FORCE_TOL
    assert o["energy"] == pytest.approx(float(z["energy"]), rel=ENERGY_TOL)
    if s.msld:
        assert rel_rms(o["lambdaForce"][1:], z["lambdaForce"][1:]) < DUDL_TOL
