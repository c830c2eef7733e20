"""FP64 CPU restatement of the reference's PME reciprocal space and Ewald
self term (test infrastructure only: tests/, the checker in smoke() and the
measurement script import it; the product never does).

Follows, in FP64 with numpy's FFT in place of cuFFT:
  * grid sizes from the grid spacing, Potential::initialize
    (src/system/potential.cxx:1204-1218): the smallest of j*{32,27,24,20,18}
    above L/spacing, j the power of two that puts L/spacing in [16j, 32j);
  * B-spline moduli 1/|b(m)|^2 per dimension (potential.cxx:1243-1290), with
    b(m) = sum_{l=1}^{n-1} M_n(l) exp(2 pi i m l / K);
  * the charge spread (getforce_ewald_spread_kernel, src/nbrecip/nbrecip.cu:
    85-213): u = x K / L, grid point (floor(u) + t) mod K receives
    lambda q M_n(u - floor(u) + n - 1 - t), t = 0..n-1, in each dimension;
  * the convolution (nbrecip.cu:215-256): the unnormalised R2C spectrum times
    B(m) (kElectric / 2 pi V) exp(-pi^2 k^2 / beta^2) / k^2, k = m / L with
    m folded to [-K/2, K/2], zero at m = 0;
  * the gather (nbrecip.cu:258-465): phi_i = sum of the unnormalised C2R grid
    times the atom's weights; E = sum_i lambda q_i phi_i; dU/dx_i =
    2 lambda q_i (K / L) sum dM ...; dU/dlambda_b = 2 sum_{i in b} q_i phi_i;
  * the self term (getforce_ewaldself_kernel, nbrecip.cu:19-55):
    E = -beta kElectric / sqrt(pi) sum (lambda q)^2, dU/dlambda_b =
    2 lambda_b (-beta kElectric / sqrt(pi)) sum_{i in b} q_i^2.
Atoms of block 0 (the environment) have lambda 1 and no dU/dlambda; block b
of an atom is the low 16 bits of its siteBlock (Msld merge_site_block,
src/msld/msld.cu:470-476).

``ewald_recip_exact`` is the plain Ewald reciprocal sum over k vectors, an
independent check that the restatement converges to the right physics.

Triclinic cells (the flagBox branch of the same kernels; the box given as the
6 floats (A_x, B_y, C_z, B_x, C_x, C_y) of a lower-triangular cell A = (A_x,
0, 0), B = (B_x, B_y, 0), C = (C_x, C_y, C_z)): the fractional coordinates
s = H^-1 x (H the cell matrix with columns A, B, C; State::kTricBox_f,
src/system/state.cxx:485-491, holds H^-1) replace x / L, so u_d = K_d s_d
(nbrecip.cu:116-178); the wave vectors are k = H^-T m (nbrecip.cu:236-242);
dU/dx = H^-T (dU/ds) (nbrecip.cu:456-462); V = A_x B_y C_z; the grid sizes
come from the edge lengths |A|, |B|, |C| (potential.cxx:1206, box.a).
"""
from __future__ import annotations

import math

import numpy as np

GOOD_SIZES = (32, 27, 24, 20, 18, 16)


def grid_size(length: float, spacing: float) -> int:
    """Grid points along one box edge (potential.cxx:1204-1218)."""
    md = np.float32(np.float32(length) / np.float32(spacing))
    j = 1
    while md >= 32 * j:
        j *= 2
    k = 0
    while k < 5 and md < j * GOOD_SIZES[k]:
        k += 1
    return j * GOOD_SIZES[k - 1]


def bspline_int(order: int) -> np.ndarray:
    """M_n(l) at integers l = 0..n (cardinal B-spline of order n)."""
    m = np.zeros(order + 1)
    m[1] = 1.0                                    # M_2(l): 0, 1, 0
    for k in range(3, order + 1):
        new = np.zeros(order + 1)
        for l in range(k + 1):
            a = m[l] if l < order + 1 else 0.0
            b = m[l - 1] if l >= 1 else 0.0
            new[l] = (l * a + (k - l) * b) / (k - 1)
        m = new
    return m


def moduli(K: int, order: int) -> np.ndarray:
    """1/|b(m)|^2 for m = 0..K-1 (potential.cxx:1243-1290)."""
    M = bspline_int(order)
    m = np.arange(K)[:, None]
    l = np.arange(1, order)[None, :]
    ph = 2 * np.pi * m * l / K
    re = (M[1:order] * np.cos(ph)).sum(1)
    im = (M[1:order] * np.sin(ph)).sum(1)
    return 1.0 / (re * re + im * im)


def weights(frac: np.ndarray, order: int):
    """w[..., t] = M_n(frac + n - 1 - t), dw = dM_n/du at the same points."""
    frac = np.asarray(frac, np.float64)
    a = np.ones(frac.shape + (1,))                # M_1(frac + j), j = 0
    prev = a
    for k in range(2, order + 1):
        prev = a
        new = np.zeros(frac.shape + (k,))
        for j in range(k):
            x = frac + j
            left = a[..., j] if j < k - 1 else 0.0
            right = a[..., j - 1] if j >= 1 else 0.0
            new[..., j] = (x * left + (k - x) * right) / (k - 1)
        a = new
    der = np.zeros(frac.shape + (order,))
    for j in range(order):                         # M_n'(x) = M_{n-1}(x) - M_{n-1}(x - 1)
        left = prev[..., j] if j < order - 1 else 0.0
        right = prev[..., j - 1] if j >= 1 else 0.0
        der[..., j] = left - right
    return a[..., ::-1], der[..., ::-1]


def atom_lambda(site_block, lam):
    """Per-atom lambda scale and block index (0 = environment, scale 1)."""
    b = np.asarray(site_block, np.int64) & 0xFFFF
    l = np.where(b > 0, np.asarray(lam, np.float64)[b], 1.0) if lam is not None else np.ones(len(b))
    return l, b


def cell(box):
    """(H, H^-1) of a box: 3 edge lengths or the 6-float triclinic cell."""
    b = np.asarray(box, np.float64).reshape(-1)
    if len(b) == 3:
        H = np.diag(b)
    else:
        H = np.array([[b[0], b[3], b[4]], [0.0, b[1], b[5]], [0.0, 0.0, b[2]]])
    return H, np.linalg.inv(H)


def edge_lengths(box):
    """|A|, |B|, |C| of a box (3 or 6 floats): the lengths the grid sizes use."""
    H, _ = cell(box)
    return np.sqrt((H * H).sum(0))


def fractional(xyz, box):
    """s = H^-1 x by back substitution (z first), FP64."""
    b = np.asarray(box, np.float64).reshape(-1)
    x = np.asarray(xyz, np.float64)
    if len(b) == 3:
        return x / b
    sz = x[:, 2] / b[2]
    sy = (x[:, 1] - b[5] * sz) / b[1]
    sx = (x[:, 0] - b[3] * sy - b[4] * sz) / b[0]
    return np.stack([sx, sy, sz], 1)


def pme_recip(xyz, q, box, K, order, beta, kElectric, site_block=None, lam=None):
    """(energy, dU/dx [N,3], dU/dlambda [L] or None, phi [N]) of one system;
    box: 3 edge lengths or the 6-float triclinic cell."""
    xyz = np.asarray(xyz, np.float64)
    q = np.asarray(q, np.float64)
    H, Hinv = cell(box)
    frac = fractional(xyz, box)
    N = len(q)
    K = [int(k) for k in K]
    if site_block is None:
        site_block = np.zeros(N, np.int64)
    l, b = atom_lambda(site_block, lam)
    qe = l * q
    W, D, idx = [], [], []
    for d in range(3):
        u = frac[:, d] * K[d]
        u0 = np.floor(u)
        w, dw = weights(u - u0, order)
        W.append(w)
        D.append(dw)
        idx.append((u0.astype(np.int64)[:, None] + np.arange(order)[None, :]) % K[d])
    ix = idx[0][:, :, None, None]
    iy = idx[1][:, None, :, None]
    iz = idx[2][:, None, None, :]
    w3 = W[0][:, :, None, None] * W[1][:, None, :, None] * W[2][:, None, None, :]
    grid = np.zeros(K)
    np.add.at(grid, (np.broadcast_to(ix, w3.shape), np.broadcast_to(iy, w3.shape),
                     np.broadcast_to(iz, w3.shape)), qe[:, None, None, None] * w3)
    F = np.fft.rfftn(grid)
    m1 = np.arange(K[0]); m1 = np.where(2 * m1 <= K[0], m1, m1 - K[0])
    m2 = np.arange(K[1]); m2 = np.where(2 * m2 <= K[1], m2, m2 - K[1])
    m3 = np.arange(K[2] // 2 + 1)
    # k = H^-T m
    mm = np.stack(np.meshgrid(m1, m2, m3, indexing="ij"), -1).astype(np.float64)
    kv = mm @ Hinv
    k2 = (kv * kv).sum(-1)
    B = (moduli(K[0], order)[:, None, None] * moduli(K[1], order)[None, :, None]
         * moduli(K[2], order)[: K[2] // 2 + 1][None, None, :])
    V = H[0, 0] * H[1, 1] * H[2, 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        G = B * (0.5 * kElectric / (np.pi * V)) * np.exp(-np.pi ** 2 * k2 / beta ** 2) / k2
    G[0, 0, 0] = 0.0
    phi_grid = np.fft.irfftn(F * G, s=K, axes=(0, 1, 2)) * (K[0] * K[1] * K[2])   # cuFFT C2R is unnormalised
    P = phi_grid[np.broadcast_to(ix, w3.shape), np.broadcast_to(iy, w3.shape), np.broadcast_to(iz, w3.shape)]
    phi = (P * w3).sum((1, 2, 3))
    gs = np.zeros((N, 3))          # dU/ds
    for d in range(3):
        parts = [W[0], W[1], W[2]]
        parts[d] = D[d]
        g3 = parts[0][:, :, None, None] * parts[1][:, None, :, None] * parts[2][:, None, None, :]
        gs[:, d] = 2 * qe * K[d] * (P * g3).sum((1, 2, 3))
    grad = gs @ Hinv               # dU/dx = H^-T dU/ds
    energy = float((qe * phi).sum())
    lforce = None
    if lam is not None:
        lforce = np.zeros(len(lam))
        np.add.at(lforce, b, np.where(b > 0, 2 * q * phi, 0.0))
    return energy, grad, lforce, phi


def ewald_self(q, beta, kElectric, site_block=None, lam=None):
    """(energy, dU/dlambda [L] or None) of getforce_ewaldself."""
    q = np.asarray(q, np.float64)
    pre = -beta * kElectric / math.sqrt(math.pi)
    if site_block is None:
        site_block = np.zeros(len(q), np.int64)
    l, b = atom_lambda(site_block, lam)
    e = pre * q * q
    energy = float((l * l * e).sum())
    lforce = None
    if lam is not None:
        lforce = np.zeros(len(lam))
        np.add.at(lforce, b, np.where(b > 0, 2 * l * e, 0.0))
    return energy, lforce


def ewald_recip_exact(xyz, q, box, beta, kElectric, kmax: int):
    """Plain Ewald reciprocal energy and dU/dx over |m_d| <= kmax (box: 3
    edge lengths or the 6-float triclinic cell; k = H^-T m)."""
    xyz = np.asarray(xyz, np.float64)
    q = np.asarray(q, np.float64)
    H, Hinv = cell(box)
    V = H[0, 0] * H[1, 1] * H[2, 2]
    r = np.arange(-kmax, kmax + 1)
    m = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    m = m[np.any(m != 0, 1)]
    k = m @ Hinv
    k2 = (k * k).sum(1)
    pref = kElectric / (2 * np.pi * V) * np.exp(-np.pi ** 2 * k2 / beta ** 2) / k2
    ph = 2 * np.pi * xyz @ k.T                      # [N, M]
    c, s = np.cos(ph), np.sin(ph)
    Sr, Si = q @ c, q @ s
    energy = float((pref * (Sr * Sr + Si * Si)).sum())
    # dE/dx_i = sum_m pref 2 (Sr dSr + Si dSi), dSr/dx_i = -q_i 2 pi k sin, dSi/dx_i = q_i 2 pi k cos
    coef = pref[None, :] * 2 * (-Sr[None, :] * s + Si[None, :] * c) * q[:, None] * 2 * np.pi
    grad = coef @ k
    return energy, grad
