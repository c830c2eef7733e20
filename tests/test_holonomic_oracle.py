"""The FP64 constraint restatement (oracle/holonomic_oracle.py): bond
lengths restored, linear momentum of every cluster unchanged, corrections
along the previous bond vectors, velocity projection; and against golden
vectors from the reference's own holonomic_position / holonomic_velocity
(src/holonomic/holonomic.cu, built unmodified; make_golden.py
--holonomic-only): SETTLE for waters, SHAKE for X-H groups."""
import glob
import os

import numpy as np
import pytest

from oracle import holonomic_oracle as H

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "holonomic_*.npz")))


def _bond_error(cl, x):
    err = 0.0
    for idx, bonds, b0 in cl:
        for (a, b), L in zip(bonds, b0):
            err = max(err, abs(np.linalg.norm(x[idx[a]] - x[idx[b]]) - L) / L)
    return err


@pytest.mark.parametrize("jitter", [0.01, 0.05])
def test_position_constraints(jitter):
    T, B1, B2, B3, xp, x, ism = H.test_clusters(seed=1, jitter=jitter)
    cl = H.clusters(T, B1, B2, B3)
    xn, v, it = H.constrain_position(cl, xp, x, ism, 0.02)
    assert it <= 8
    assert _bond_error(cl, xn) < 1e-12
    m = 1 / ism[0::3] ** 2
    for idx, bonds, _ in cl:
        idx = np.asarray(idx)
        assert np.abs(((xn[idx] - x[idx]) * m[idx, None]).sum(0)).max() < 1e-12
        # the correction of each atom lies in the span of the previous bond vectors
        dp = np.array([xp[idx[a]] - xp[idx[b]] for a, b in bonds])
        for a in range(len(idx)):
            res = np.linalg.lstsq(dp.T, xn[idx[a]] - x[idx[a]], rcond=None)[1]
            assert res.size == 0 or res[0] < 1e-20
    assert np.allclose(v, (xn - xp) / 0.02 * np.isin(np.arange(len(x)), np.concatenate([c[0] for c in cl]))[:, None])


def test_velocity_constraints():
    T, B1, B2, B3, xp, x, ism = H.test_clusters(seed=2)
    cl = H.clusters(T, B1, B2, B3)
    v0 = np.random.default_rng(0).normal(size=xp.shape)
    v = H.constrain_velocity(cl, xp, v0, ism)
    m = 1 / ism[0::3] ** 2
    for idx, bonds, _ in cl:
        for a, b in bonds:
            assert abs((v[idx[a]] - v[idx[b]]) @ (xp[idx[a]] - xp[idx[b]])) < 1e-12
        idx = np.asarray(idx)
        assert np.allclose((v[idx] * m[idx, None]).sum(0), (v0[idx] * m[idx, None]).sum(0), atol=1e-12)


def test_files_present():
    assert len(FILES) == 2


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_oracle_matches_reference(path):
    z = np.load(path)
    T = z["tri"].view(H.TRI_DTYPE)
    B1, B2, B3 = z["b1"].view(H.B1_DTYPE), z["b2"].view(H.B2_DTYPE), z["b3"].view(H.B3_DTYPE)
    cl = H.clusters(T, B1, B2, B3)
    xn, v, _ = H.constrain_position(cl, z["x_prev"], z["x"], z["ism"], float(z["halfdt"]))
    # the reference: SETTLE (waters) and SHAKE to 1e-10 (X-H), FP32 inverse masses and velocities
    assert np.abs(xn - z["x_ref"]).max() < 1e-7
    assert np.sqrt(((v - z["v_ref"]) ** 2).sum() / (z["v_ref"] ** 2).sum()) < 1e-5
    vp = H.constrain_velocity(cl, z["x_ref"], z["v_in"], z["ism"].astype(np.float32))
    assert np.sqrt(((vp - z["v_proj_ref"]) ** 2).sum() / (z["v_proj_ref"] ** 2).sum()) < 1e-5
