"""The FP64 oracle on the reference's own CHARMM fixtures -- test/water216
(216 TIP3P waters, minimized coordinates, par_all36_prot + par_water_ions)
and test/newDHFR (dihydrofolate reductase in water, 23,558 atoms, 35 LJ
types, par_all22_prot) -- against the reference's own CUDA direct space,
nb14/nbex pair lists and PME built unmodified (golden vectors made by
tests/golden/make_golden.py: fixture_<name>.npz holds the system as
oracle/charmm.py read it from the PSF/CRD/parameter files, real_<name>.npz
the reference's outputs).  DHFR runs with its own input's settings (rcut 9,
rswitch 7.5, beta 0.32, PME order 4 on a 64^3 grid); its LJ table has 35
types, so the CUDA path uses the per-pair table, not the combination rule."""
import os

import numpy as np
import pytest

import oracle
from blade_b200 import systems
from oracle import pme_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["water216", "dhfr"]
FORCE_TOL = 5e-6      # relative RMS of dU/dx: the reference computes in FP32
ENERGY_TOL = 5e-6     # energy difference per max(|E|, N)
PME_FORCE_TOL = 3e-5  # FP32 grid sums of 23,558 atoms in the reference
K_ELECTRIC = 332.0716


def load(name):
    s = systems.load_fixture(os.path.join(HERE, "golden", f"fixture_{name}.npz"))
    return s, np.load(os.path.join(HERE, "golden", f"real_{name}.npz"))


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def energy_ok(e, ref, n, tol=ENERGY_TOL):
    return abs(e - ref) <= tol * max(abs(ref), n)


@pytest.mark.parametrize("name", NAMES)
def test_fixture_contents(name):
    s, _ = load(name)
    assert s.N == {"water216": 648, "dhfr": 23558}[name]
    assert s.nTypes == {"water216": 2, "dhfr": 35}[name]
    assert abs(float(s.nbonds["q"].sum()) - {"water216": 0.0, "dhfr": -11.0}[name]) < 1e-3
    e = set(map(tuple, s.excl.tolist()))
    assert all((j, i) in e for i, j in s.excl.tolist())
    # every 1-4 pair is excluded from the direct space; nbex holds the other exclusions
    assert all((int(i), int(j)) in e for i, j in s.nb14["idx"])
    assert len(s.nbex) + len(s.nb14) == len(s.excl) // 2


@pytest.mark.parametrize("name", NAMES)
def test_direct_space_matches_reference(name):
    s, z = load(name)
    o = oracle.nbdirect(s)
    assert rel_rms(o["grad"], z["grad"].astype(np.float64)) <= FORCE_TOL
    assert energy_ok(o["energy"], float(z["energy"]), s.N)


@pytest.mark.parametrize("name", NAMES)
def test_pair_lists_match_reference(name):
    s, z = load(name)
    if len(s.nb14):
        o = oracle.pair_lists(s, which="nb14")
        assert rel_rms(o["grad"], z["grad14"].astype(np.float64)) <= FORCE_TOL
        assert energy_ok(o["energy"], float(z["energy14"]), s.N)
    o = oracle.pair_lists(s, which="nbex")
    assert rel_rms(o["grad"], z["gradex"].astype(np.float64)) <= FORCE_TOL
    assert energy_ok(o["energy"], float(z["energyex"]), s.N)


@pytest.mark.parametrize("name", NAMES)
def test_pme_matches_reference(name):
    s, z = load(name)
    K = [int(k) for k in z["K"]]
    E, g, _, _ = pme_oracle.pme_recip(s.xyz, s.nbonds["q"], s.box, K, int(z["order"]), s.betaEwald, K_ELECTRIC)
    assert rel_rms(g, z["gradpme"].astype(np.float64)) <= PME_FORCE_TOL
    assert energy_ok(E, float(z["energypme"]), s.N)
    Es, _ = pme_oracle.ewald_self(s.nbonds["q"], s.betaEwald, K_ELECTRIC)
    assert Es == pytest.approx(float(z["energyself"]), rel=1e-6)
