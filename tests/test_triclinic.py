"""Triclinic cells (State::typeBox, the reference's flagBox branch of the
direct-space path): the CPU restatement of the list wraps atoms into the
brick A_x x B_y x C_z (src/main/real3.h:340-360) and culls over half-shell
images centred under the shear (src/domdec/cull.cu:141-190); the FP64 oracle
sums every pair over lattice images.  Checked here: the list's active tiles
hold every pair within rCut exactly once, an orthorhombic cell given as a
triclinic one (zero off-diagonal terms) builds the identical list, and the
oracle's forces follow the lattice (translating every atom by a cell vector
changes nothing)."""
import dataclasses

import numpy as np
import pytest

import oracle
from blade_b200 import systems


def _tiles_pairs(s, L, rc):
    """(set of atom pairs evaluated, number evaluated) by walking the active
    tiles of the list the way the pair kernel does."""
    B = L["blockCount"]
    packed, bmin, bmax = oracle.pack(L, s.xyz, s.box6())
    table = oracle.shift_table(s.box6()).astype(np.float64)
    active = oracle.active_tiles(L, bmin, bmax, s.box6(), rc)
    slot = L["slotAtom"].reshape(B, 32)
    P = packed.reshape(B, 32, 3).astype(np.float64)
    excl = set(map(tuple, s.excl.tolist()))
    seen, n = set(), 0
    for i in range(B):
        for c in range(L["candStart"][i], L["candStart"][i + 1]):
            if not active[c]:
                continue
            j, code = (int(v) for v in L["cand"][c])
            d = P[i][:, None, :] - (P[j][None, :, :] + table[code])
            r2 = (d * d).sum(-1)
            ok = (r2 < rc * rc) & (slot[i][:, None] >= 0) & (slot[j][None, :] >= 0)
            if i == j and code == 0:
                ok &= np.arange(32)[None, :] > np.arange(32)[:, None]
            for li, lj in zip(*np.nonzero(ok)):
                a, b = int(slot[i][li]), int(slot[j][lj])
                if (a, b) in excl:
                    continue
                seen.add((min(a, b), max(a, b)))
                n += 1
    return seen, n


def test_every_pair_exactly_once_triclinic():
    s = systems.water_box_tric()
    L = oracle.build_list(s)
    seen, n = _tiles_pairs(s, L, s.rCut)
    o = oracle.nbdirect(s)
    assert n == len(seen)                 # no pair twice
    assert n == o["pairs"]                # none missing (FP64 count of the oracle)


def test_orthorhombic_cell_as_triclinic_builds_the_same_list():
    s = systems.water_box()
    t = dataclasses.replace(s, tric=np.zeros(3, np.float32))
    a, b = oracle.build_list(s), oracle.build_list(t)
    for k in ("wrap", "sortedAtom", "slotAtom", "bmin", "bmax", "cand", "candExcl", "masks"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(oracle.shift_table(s.box), oracle.shift_table(t.box6()))


def test_shift_table_centres_the_shear():
    s = systems.water_box_tric()
    table = oracle.shift_table(s.box6())
    # every image of the half shell except the own image is a nonzero lattice vector,
    # and the sheared images stay within one brick edge of the origin in x and y
    ax, by, cz = s.box
    assert np.allclose(table[0], 0)
    assert (np.abs(table[1:, 0]) <= 1.5 * ax + 1e-3).all()
    assert (np.abs(table[1:, 1]) <= 1.5 * by + 1e-3).all()


def test_oracle_is_lattice_periodic():
    s = systems.water_box_tric()
    o = oracle.nbdirect(s)
    A = np.array([s.box[0], 0, 0]); C = np.array([s.tric[1], s.tric[2], s.box[2]])
    x = s.xyz.astype(np.float64)
    x[::7] += A
    x[3::11] -= C
    o2 = oracle.nbdirect(s, xyz=x)
    assert o2["pairs"] == o["pairs"]
    assert np.abs(o2["grad"] - o["grad"]).max() < 1e-8
    assert o2["energy"] == pytest.approx(o["energy"], rel=1e-12)


GOLDEN = ["water_tric", "msld_tric"]


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_matches_reference_triclinic(name):
    """Against the reference's own triclinic direct space (flagBox = true,
    tests/golden/make_golden.py --tric-only)."""
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    from test_gpu_triclinic import CASES
    z = np.load(os.path.join(here, "golden", f"tric_{name}.npz"))
    s = CASES[name]()
    assert np.array_equal(s.xyz, z["xyz"])
    assert np.array_equal(s.tric_box(), z["tric_box"])
    o = oracle.nbdirect(s)
    g = z["grad"].astype(np.float64)
    assert np.sqrt(((o["grad"] - g) ** 2).sum() / (g ** 2).sum()) <= 5e-6
    assert abs(o["energy"] - float(z["energy"])) <= 5e-6 * max(abs(o["energy"]), s.N)
    if s.msld is not None:
        lf = z["lambdaForce"]
        assert np.abs(o["lambdaForce"][1:] - lf[1:]).max() <= 1e-5 * max(1.0, np.abs(lf).max())


@pytest.mark.parametrize("name", GOLDEN)
def test_pme_oracle_matches_reference_triclinic(name):
    """The FP64 PME restatement in a triclinic cell against the reference's
    own triclinic getforce_ewald (flagBox = true with State::kTricBox_f;
    tests/golden/make_golden.py --tric-pme-only)."""
    import os
    import sys
    from oracle import pme_oracle
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    from test_gpu_triclinic import CASES
    z = np.load(os.path.join(here, "golden", f"tric_pme_{name}.npz"))
    s = CASES[name]()
    assert np.array_equal(s.xyz, z["xyz"]) and np.array_equal(s.tric_box(), z["tric_box"])
    K = [int(k) for k in z["K"]]
    assert K == [pme_oracle.grid_size(L, 1.0) for L in pme_oracle.edge_lengths(s.box6())]
    lam = s.lambdas() if s.msld is not None else None
    E, g, lf, _ = pme_oracle.pme_recip(s.xyz, s.nbonds["q"], s.box6(), K, int(z["order"]), s.betaEwald, 332.0716,
                                       s.nbonds["siteBlock"], lam)
    zg = z["grad"].astype(np.float64)
    assert np.sqrt(((g - zg) ** 2).sum() / (zg ** 2).sum()) <= 1e-5      # the reference computes in FP32
    assert E == pytest.approx(float(z["energy"]), rel=5e-6)
    if lf is not None:
        zl = z["lambdaForce"]
        assert np.abs(lf[1:] - zl[1:]).max() <= 1e-5 * max(1.0, np.abs(zl).max())
