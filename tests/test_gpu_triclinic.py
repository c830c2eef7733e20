"""Triclinic cells on the GPU (bnb_set_box_type; the reference's flagBox
path of getforce_nbdirect, Domdec's cull and wrap): the block list equals the
CPU restatement bit for bit, forces and energies match the FP64 oracle (which
sums every lattice image) and the reference's own triclinic CUDA path
(tests/golden/tric_*.npz), the result does not change when atoms are moved by
cell vectors, and PME, which is orthorhombic here, refuses the cell."""
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


def test_pme_refuses_triclinic(cuda):
    s = systems.water_box_tric()
    nb = NbDirect(s)
    with pytest.raises(_lib.BnbError, match="unsupported"):
        nb.set_pme(order=6)
    nb.close()


GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "tric_*.npz")))


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
