"""The compiled drop-in: the reference (BLaDE) built from its own sources,
once unmodified and once with getforce_nbdirect and Domdec replaced by the
libbnb binding of oracle/dropin/bnb_dropin.cu (oracle/dropin/Makefile), runs
`run energy` on its own fixtures -- test/water216 and test/newDHFR, read
through its own parser, structure and parameter code and Potential::initialize
-- and both print their energy terms (display_nrg, src/io/io.cxx:386-395).
The direct-space term eenbdirect must agree; every other term comes from the
same reference code in both builds and must agree to the resolution of the
printed value: the reference sums its PME charge grid and its energies with
floating-point atomics, so even two runs of the unmodified program can differ
in the last printed digit."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "oracle", "_ref", "dropin")
TERMS = ["bond", "angle", "urey", "dihe", "impr", "cmap", "nb14", "nbdirect", "nbrecip", "nbrecipself",
         "nbrecipexcl", "lambda", "theta", "cats", "noe", "harmonic", "mmfp", "resd", "mlp", "bias", "potential",
         "kinetic", "total"]                      # EETerm order, src/system/potential.h:20-44
NBDIRECT = TERMS.index("nbdirect")
SUMS = {TERMS.index(t) for t in ("potential", "total", "nbdirect")}
ENERGY_TOL = 1e-5                                 # eenbdirect difference per max(|E|, atoms)
PRINT_TOL = 1e-4                                  # one unit of the last printed digit (display_nrg, %.4f)
ATOMIC_TOL = 2e-7                                 # relative: FP32 atomic summation order in the reference
CASES = {"water216": ("energy_water216.inp", 648), "dhfr": ("energy_dhfr.inp", 23558)}


def _energies(binary, script, tmp_path):
    env = dict(os.environ, OMP_NUM_THREADS="1")   # BLaDE runs one GPU per OpenMP thread
    r = subprocess.run([binary, script], cwd=tmp_path, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for line in reversed(r.stdout.splitlines()):
        parts = line.split()
        if len(parts) == len(TERMS):
            try:
                return np.array([float(p) for p in parts])
            except ValueError:
                continue
    raise AssertionError("no energy line in the output:\n" + r.stdout[-2000:])


@pytest.mark.parametrize("case", list(CASES))
def test_patched_reference_matches_unpatched(cuda, case, tmp_path):
    ref, bnb = os.path.join(OUT, "blade_ref"), os.path.join(OUT, "blade_bnb")
    if not (os.path.exists(ref) and os.path.exists(bnb)):
        pytest.skip("reference builds not present (oracle/dropin/Makefile needs the reference sources)")
    name, atoms = CASES[case]
    text = open(os.path.join(ROOT, "oracle", "dropin", name)).read().replace("@FIX@", os.path.join(OUT, "fixtures"))
    script = tmp_path / name
    script.write_text(text)
    e_ref = _energies(ref, str(script), tmp_path)
    e_bnb = _energies(bnb, str(script), tmp_path)
    assert e_ref[NBDIRECT] != 0.0
    assert abs(e_bnb[NBDIRECT] - e_ref[NBDIRECT]) <= ENERGY_TOL * max(abs(e_ref[NBDIRECT]), atoms), \
        (e_bnb[NBDIRECT], e_ref[NBDIRECT])
    for k in range(len(TERMS)):
        if k not in SUMS:
            assert abs(e_bnb[k] - e_ref[k]) <= PRINT_TOL + ATOMIC_TOL * abs(e_ref[k]), (TERMS[k], e_bnb[k], e_ref[k])
