"""Lambda trajectories in the reference's .lmd format and the flattening
histograms taken from them.

BLaDE writes the lambda of every non-environment block every freqLMD steps
(``print_lmd``, src/io/io.cxx:347-371): as text, one line per frame with the
step in ``%10ld`` followed by `` %8.6f`` per block; or as XDR, per frame the
block count (4-byte big-endian int) followed by that many 4-byte big-endian
floats.  ALF reads these files to build its histograms; ``histograms`` builds
the same statistics that ``bnb_lambda_histogram`` accumulates on the GPU, so
a trajectory written here (or by the reference) feeds ``blade_b200.alf``.
"""
from __future__ import annotations

import struct

import numpy as np


def write_lmd(path: str, steps, lam: np.ndarray, binary: bool = False):
    """lam: [frames, L] with block 0 (environment) first; writes blocks 1..L-1."""
    lam = np.asarray(lam)
    with open(path, "wb" if binary else "w") as f:
        for step, row in zip(steps, lam):
            if binary:
                f.write(struct.pack(">i", lam.shape[1] - 1))
                f.write(np.asarray(row[1:], ">f4").tobytes())
            else:
                f.write("%10ld" % int(step) + "".join(" %8.6f" % float(v) for v in row[1:]) + "\n")


def read_lmd(path: str, binary: bool = False):
    """(steps or None, lam [frames, L-1]) -- the text form carries steps, XDR does not."""
    if not binary:
        rows = [line.split() for line in open(path) if line.strip()]
        steps = np.array([int(r[0]) for r in rows], np.int64)
        return steps, np.array([[float(v) for v in r[1:]] for r in rows], np.float64)
    data = open(path, "rb").read()
    frames, off = [], 0
    while off < len(data):
        (n,) = struct.unpack_from(">i", data, off)
        off += 4
        frames.append(np.frombuffer(data, ">f4", n, off).astype(np.float64))
        off += 4 * n
    return None, np.array(frames)


def histograms(lam: np.ndarray, pairs: np.ndarray, fixed=None):
    """Flattening statistics of a trajectory lam [frames, L] (block 0 first):
    (hist1 [L,32], hist2 [P,8,8], endCount [L]) binned exactly as
    bnb_lambda_histogram does (bin = min(int(lambda*32), 31), lambda > 0.99)."""
    lam = np.asarray(lam, np.float64)
    F, L = lam.shape
    fixed = np.zeros(L, bool) if fixed is None else np.asarray(fixed, bool)
    b1 = np.clip((lam * 32).astype(np.int64), 0, 31)
    h1 = np.zeros((L, 32), np.int64)
    for i in range(L):
        if not fixed[i]:
            h1[i] = np.bincount(b1[:, i], minlength=32)
    end = np.where(fixed, 0, (lam > 0.99).sum(0))
    h2 = np.zeros((len(pairs), 8, 8), np.int64)
    b8 = np.clip((lam * 8).astype(np.int64), 0, 7)
    for p, (i, j) in enumerate(pairs):
        np.add.at(h2[p], (b8[:, i], b8[:, j]), 1)
    return h1, h2, end.astype(np.int64)
