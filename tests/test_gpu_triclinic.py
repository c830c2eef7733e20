"""Triclinic cells on the GPU (bnb_set_box_type; the reference's flagBox
path of getforce_nbdirect, Domdec's cull and wrap): the block list equals the
CPU restatement bit for bit, forces and energies match the FP64 oracle (which
sums every lattice image) and the reference's own triclinic CUDA path
(tests/golden/tric_*.npz), the result does not change when atoms are moved by
cell vectors; PME reciprocal space in the cell (the flagBox branch of
getforce_ewald) matches the FP64 oracle, the reference's own triclinic PME
(tests/golden/tric_pme_*.npz) and is unchanged by cell-vector moves."""
import dataclasses
import glob
import os

import numpy as np
import pytest
import torch

import oracle
from blade_b200 import _lib, systems
from blade_b200.nbdirect import NbDirect

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FORCE_TOL = 1e-5      # relative RMS of dU/dx vs the FP64 oracle
ENERGY_TOL = 1e-5     # per max(|E|, N)
REF_FORCE_TOL = 1e-5  # vs the reference's FP32 build


def _msld_tric():
    """The triclinic water box with its first 60 waters as two MSLD sites."""
    s = systems.water_box_tric()
    m = systems.msld_water()
    nb = s.nbonds.copy()
    blocks = np.zeros(s.N, np.int32)
    for k in range(4):                         # site 1: blocks 1-2, site 2: blocks 3-4
        site = 1 + k // 2
        atoms = np.arange(3 * 15 * k, 3 * 15 * (k + 1))
        nb["siteBlock"][atoms] = (site << 16) | (k + 1)
        blocks[atoms] = k + 1
    excl = [s.excl]
    for a, b in ((1, 2), (3, 4)):              # substituents of one site do not see each other
        ia, ib = np.nonzero(blocks == a)[0], np.nonzero(blocks == b)[0]
        pairs = np.stack(np.meshgrid(ia, ib, indexing="ij"), -1).reshape(-1, 2)
        excl += [pairs, pairs[:, ::-1]]
    ms = systems.Msld(5, 3, np.array([0, 1, 3, 5], np.int32), np.array([0, 1, 1, 2, 2], np.int32),
                      np.array([0.0, 0.4, -0.3, 0.9, 0.1]))
    return dataclasses.replace(s, nbonds=nb, excl=np.unique(np.concatenate(excl).astype(np.int32), axis=0),
                               msld=ms, name="msld_tric")


CASES = {"water_tric": systems.water_box_tric, "msld_tric": _msld_tric}


def _rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("case", list(CASES))
def test_list_bitexact_and_forces_match_oracle(cuda, case):
    s = CASES[case]()
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    g = nb.get_list()
    o = oracle.build_list(s)
    for k in ("wrap", "blockBounds", "sortedAtom", "slotAtom", "bmin", "bmax", "candStart", "cand",
              "candExcl", "masks"):
        assert np.array_equal(g[k], o[k]), k
    nb.set_counting(True)
    f, lf, e = nb.evaluate(pos)
    torch.cuda.synchronize()
    assert nb.status() == 0
    ref = oracle.nbdirect(s)
    assert nb.pair_count() == ref["pairs"]
    assert _rel(f.cpu().numpy(), ref["grad"]) <= FORCE_TOL
    assert abs(float(e[0]) - ref["energy"]) <= ENERGY_TOL * max(abs(ref["energy"]), s.N)
    if s.msld is not None:
        l = lf.cpu().numpy()
        assert np.abs(l[1:] - ref["lambdaForce"][1:]).max() <= 1e-5 * max(1.0, np.abs(ref["lambdaForce"]).max())
    nb.close()


def test_lattice_translations_change_nothing(cuda):
    s = systems.water_box_tric()
    A = np.array([s.box[0], 0, 0], np.float32)
    B = np.array([s.tric[0], s.box[1], 0], np.float32)
    C = np.array([s.tric[1], s.tric[2], s.box[2]], np.float32)
    x2 = s.xyz.copy()
    x2[::5] += A
    x2[1::7] -= B
    x2[2::9] += C
    nb = NbDirect(s)
    out = []
    for x in (s.xyz, x2):
        pos = nb.positions_tensor([x])
        nb.update_domdec(pos, True)
        f, _, e = nb.evaluate(pos)
        torch.cuda.synchronize()
        out.append((f.cpu().numpy(), float(e[0])))
    # the same physics; only the FP32 rounding of the moved coordinates differs
    assert _rel(out[1][0], out[0][0]) <= 1e-5
    assert abs(out[0][1] - out[1][1]) <= 1e-6 * s.N
    nb.close()


PME_FORCE_TOL = 2e-5      # relative RMS of dU/dx vs FP64 (FP32 B-splines and FFT)
PME_REF_FORCE_TOL = 1e-4  # against the reference's FP32 build
K_ELECTRIC = 332.0716


def _pme_case(name):
    s = CASES[name]()
    from oracle import pme_oracle
    K = tuple(pme_oracle.grid_size(L, 1.0) for L in pme_oracle.edge_lengths(s.box6()))
    return s, K


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("order", [4, 6])
def test_pme_matches_oracle(cuda, name, order):
    from oracle import pme_oracle
    s, K = _pme_case(name)
    nb = NbDirect(s)
    nb.set_pme(order=order, grid_space=1.0)
    assert nb.pme_grid(0) == K
    f, lf, e = nb.evaluate_pme()
    lam = s.lambdas() if s.msld else None
    E, g, L, _ = pme_oracle.pme_recip(s.xyz, s.nbonds["q"], s.box6(), K, order, s.betaEwald, K_ELECTRIC,
                                      s.nbonds["siteBlock"], lam)
    assert _rel(f.cpu().numpy(), g) < PME_FORCE_TOL
    assert float(e.cpu()[0]) == pytest.approx(E, rel=1e-5)
    if L is not None:
        assert np.abs(lf.cpu().numpy() - L).max() <= 2e-5 * max(1.0, np.abs(L).max())
    nb.close()


def test_pme_invariant_under_cell_vector_moves(cuda):
    s, K = _pme_case("water_tric")
    ax, bx, by, cx, cy, cz = (float(v) for v in s.tric_box())
    cellv = np.array([[ax, 0, 0], [bx, by, 0], [cx, cy, cz]])
    rng = np.random.default_rng(3)
    moved = s.xyz.astype(np.float64).copy()
    for w in range(s.N // 3):  # whole waters by random lattice translations
        moved[3 * w:3 * w + 3] += rng.integers(-2, 3, 3) @ cellv
    out = []
    for xyz in (s.xyz, moved.astype(np.float32)):
        nb = NbDirect(dataclasses.replace(s, xyz=xyz))
        nb.set_pme(order=6, grid_space=1.0)
        f, _, e = nb.evaluate_pme()
        out.append((f.cpu().numpy(), float(e.cpu()[0])))
        nb.close()
    assert _rel(out[1][0], out[0][0]) <= 1e-5
    assert out[1][1] == pytest.approx(out[0][1], rel=1e-5)


PME_GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "tric_pme_*.npz")))


@pytest.mark.parametrize("path", PME_GOLDEN, ids=[os.path.basename(p)[:-4] for p in PME_GOLDEN])
def test_pme_matches_reference_triclinic_golden(cuda, path):
    z = np.load(path)
    s, K = _pme_case(str(z["case"]))
    assert np.array_equal(s.xyz, z["xyz"]) and tuple(z["K"]) == K
    nb = NbDirect(s)
    nb.set_pme(order=int(z["order"]), grid=K)
    f, lf, e = nb.evaluate_pme()
    assert _rel(f.cpu().numpy(), z["grad"].astype(np.float64)) <= PME_REF_FORCE_TOL
    assert float(e.cpu()[0]) == pytest.approx(float(z["energy"]), rel=1e-5)
    nb.close()


GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "tric_[!p]*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_matches_reference_triclinic_golden(cuda, path):
    z = np.load(path)
    s = CASES[str(z["case"])]()
    assert np.array_equal(s.xyz, z["xyz"])
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    f, lf, e = nb.evaluate(pos)
    torch.cuda.synchronize()
    assert _rel(f.cpu().numpy(), z["grad"].astype(np.float64)) <= REF_FORCE_TOL
    assert abs(float(e[0]) - float(z["energy"])) <= ENERGY_TOL * max(abs(float(z["energy"])), s.N)
    nb.close()
