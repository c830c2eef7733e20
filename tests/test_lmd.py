"""The .lmd lambda-trajectory format (src/io/io.cxx:347-371) and the
flattening histograms built from it."""
import struct

import numpy as np

from blade_b200 import lmd


def _traj(rng, F=40, L=9):
    lam = rng.dirichlet(np.ones(L - 1), F)
    return np.concatenate([np.ones((F, 1)), lam], 1)


def test_text_format_matches_reference_printf(tmp_path):
    lam = np.array([[1.0, 0.25, 0.75], [1.0, 1.0, 0.0]])
    p = tmp_path / "a.lmd"
    lmd.write_lmd(str(p), [10, 20], lam)
    assert p.read_text().splitlines() == ["        10 0.250000 0.750000", "        20 1.000000 0.000000"]
    steps, back = lmd.read_lmd(str(p))
    assert steps.tolist() == [10, 20]
    np.testing.assert_array_equal(back, lam[:, 1:])


def test_xdr_round_trip(tmp_path):
    lam = _traj(np.random.default_rng(0))
    p = tmp_path / "a.xlmd"
    lmd.write_lmd(str(p), range(len(lam)), lam, binary=True)
    raw = p.read_bytes()
    assert struct.unpack_from(">i", raw, 0)[0] == lam.shape[1] - 1
    assert len(raw) == len(lam) * 4 * lam.shape[1]
    _, back = lmd.read_lmd(str(p), binary=True)
    np.testing.assert_array_equal(back, lam[:, 1:].astype(np.float32))


def test_histograms_match_direct_count():
    rng = np.random.default_rng(1)
    lam = _traj(rng)
    lam[0, 1] = 1.0
    lam[1, 2] = 0.99
    pairs = np.array([[1, 2], [3, 8], [2, 5]])
    fixed = np.zeros(lam.shape[1], bool)
    fixed[0] = True
    h1, h2, end = lmd.histograms(lam, pairs, fixed)
    for i in range(1, lam.shape[1]):
        for f in range(len(lam)):
            assert h1[i, min(int(lam[f, i] * 32), 31)] > 0
        assert h1[i].sum() == len(lam)
        assert end[i] == (lam[:, i] > 0.99).sum()
    assert h1[0].sum() == 0 and end[0] == 0
    for p, (i, j) in enumerate(pairs):
        assert h2[p].sum() == len(lam)
        a, b = min(int(lam[5, i] * 8), 7), min(int(lam[5, j] * 8), 7)
        assert h2[p, a, b] > 0
