"""FP64 CPU restatement of the holonomic bond constraints (test
infrastructure only: tests/ and the golden-vector script import it).

The constraint problem is the reference's (holonomic_position /
holonomic_velocity, src/holonomic/holonomic.cu:238-758, clusters of
src/system/potential.h:120-138): after a drift from xPrev to x, find
multipliers lambda_c such that
    x'_a = x_a + sum_c lambda_c s(a, c) (xPrev_pa(c) - xPrev_pb(c)) / m_a
satisfies |x'_pa(c) - x'_pb(c)| = b0_c for every bond c of the cluster
(s = +1 for the first atom of the bond, -1 for the second), then
v = (x' - xPrev) / halfdt.  Solved here by Newton iteration on the full
constraint matrix to 1e-13 relative, which the reference's SETTLE
(triangles) and SHAKE (branches) approximate to their tolerance.  The
velocity constraint solves the linear system that removes the relative
velocity along every bond.
"""
from __future__ import annotations

import numpy as np

TRI_DTYPE = np.dtype([("idx", "<i4", 3), ("b0", "<f4", 3)])
B1_DTYPE = np.dtype([("idx", "<i4", 2), ("b0", "<f4", 1)])
B2_DTYPE = np.dtype([("idx", "<i4", 3), ("b0", "<f4", 2)])
B3_DTYPE = np.dtype([("idx", "<i4", 4), ("b0", "<f4", 3)])


def clusters(tri=(), b1=(), b2=(), b3=()):
    """(atom indices, bond pairs as local indices, b0) of every cluster."""
    out = []
    for t in tri:
        out.append((list(t["idx"]), [(0, 1), (0, 2), (1, 2)], [float(v) for v in t["b0"]]))
    for arr in (b1, b2, b3):
        for t in arr:
            n = len(t["idx"]) - 1
            out.append((list(t["idx"]), [(0, k + 1) for k in range(n)], [float(v) for v in t["b0"]]))
    return out


def constrain_position(cl, xPrev, x, ism, halfdt, tol=1e-13, max_iter=50):
    """Returns (x', v for the cluster atoms written into copies of x and a
    velocity array, iterations).  xPrev, x: [N,3]; ism: [3N] or [N]."""
    xPrev = np.asarray(xPrev, np.float64).reshape(-1, 3)
    x = np.array(x, np.float64).reshape(-1, 3)
    ism = np.asarray(ism, np.float64).reshape(-1)
    ism3 = ism[0::3] if len(ism) == 3 * len(x) else ism
    v = np.zeros_like(x)
    worst = 0
    for idx, bonds, b0 in cl:
        idx = np.asarray(idx)
        im = ism3[idx] ** 2
        xp = xPrev[idx]
        xc = x[idx].copy()
        dp = np.array([xp[a] - xp[b] for a, b in bonds])
        b02 = np.array(b0) ** 2
        S = np.zeros((len(idx), len(bonds)))
        for c, (a, b) in enumerate(bonds):
            S[a, c] += 1.0
            S[b, c] -= 1.0
        it = 0
        for it in range(max_iter):
            d = np.array([xc[a] - xc[b] for a, b in bonds])
            r = b02 - (d * d).sum(1)
            if np.all(np.abs(r) <= tol * b02):
                break
            # d(|d_c|^2)/d(lambda_c') = 2 d_c . (S[a_c,c'] im[a_c] - S[b_c,c'] im[b_c]) dp_c'
            A = np.zeros((len(bonds), len(bonds)))
            for c, (a, b) in enumerate(bonds):
                for cp in range(len(bonds)):
                    A[c, cp] = 2.0 * (d[c] @ dp[cp]) * (S[a, cp] * im[a] - S[b, cp] * im[b])
            lam = np.linalg.solve(A, r)
            xc += (S * im[:, None]) @ (lam[:, None] * dp)
        worst = max(worst, it)
        x[idx] = xc
        v[idx] = (xc - xp) / halfdt
    return x, v, worst


def constrain_velocity(cl, x, v, ism):
    x = np.asarray(x, np.float64).reshape(-1, 3)
    v = np.array(v, np.float64).reshape(-1, 3)
    ism = np.asarray(ism, np.float64).reshape(-1)
    ism3 = ism[0::3] if len(ism) == 3 * len(x) else ism
    for idx, bonds, _ in cl:
        idx = np.asarray(idx)
        im = ism3[idx] ** 2
        xc, vc = x[idx], v[idx].copy()
        d = np.array([xc[a] - xc[b] for a, b in bonds])
        S = np.zeros((len(idx), len(bonds)))
        for c, (a, b) in enumerate(bonds):
            S[a, c] += 1.0
            S[b, c] -= 1.0
        r = -np.array([(vc[a] - vc[b]) @ d[c] for c, (a, b) in enumerate(bonds)])
        A = np.zeros((len(bonds), len(bonds)))
        for c, (a, b) in enumerate(bonds):
            for cp in range(len(bonds)):
                A[c, cp] = (d[c] @ d[cp]) * (S[a, cp] * im[a] - S[b, cp] * im[b])
        lam = np.linalg.solve(A, r)
        v[idx] = vc + (S * im[:, None]) @ (lam[:, None] * d)
    return v


def test_clusters(seed: int = 0, n_water: int = 64, n_each: int = 16, jitter: float = 0.03):
    """Synthetic constraint problem: rigid TIP3P waters (triangles) and
    X-H groups (OH, NH2, CH3: branches 1-3) at random orientations, then
    every atom displaced by N(0, jitter) as a drift would.  Returns
    (tri, b1, b2, b3, xPrev [N,3], x [N,3], ism [3N])."""
    rng = np.random.default_rng(seed)
    pos, mass = [], []
    tri, b1, b2, b3 = [], [], [], []

    def rot():
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        a, b, c, d = q
        return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                         [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                         [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])

    def place(local, masses):
        c = rng.uniform(0, 30, 3)
        R = rot()
        i0 = len(pos)
        for p, m in zip(local, masses):
            pos.append(c + R @ np.asarray(p))
            mass.append(m)
        return i0

    roh, hh = 0.9572, 1.5139
    ang = np.arccos(1 - hh * hh / (2 * roh * roh))
    w = [(0, 0, 0), (roh, 0, 0), (roh * np.cos(ang), roh * np.sin(ang), 0)]
    for _ in range(n_water):
        i = place(w, (15.9994, 1.008, 1.008))
        tri.append(((i, i + 1, i + 2), (roh, roh, hh)))
    tet = np.array([(1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1)]) / np.sqrt(3)
    for nh, heavy, mh, bl, dst in ((1, 15.999, 1.008, 0.96, b1), (2, 14.007, 1.008, 1.01, b2),
                                   (3, 12.011, 1.008, 1.09, b3)):
        for _ in range(n_each):
            local = [(0, 0, 0)] + [tuple(bl * tet[k]) for k in range(nh)]
            i = place(local, [heavy] + [mh] * nh)
            dst.append((tuple(range(i, i + nh + 1)), (bl,) * nh))
    xPrev = np.array(pos)
    x = xPrev + rng.normal(0, jitter, xPrev.shape)
    ism = np.repeat(1.0 / np.sqrt(np.array(mass)), 3)
    T = np.array(tri, dtype=TRI_DTYPE)
    B1 = np.array(b1, dtype=B1_DTYPE)
    B2 = np.array(b2, dtype=B2_DTYPE)
    B3 = np.array(b3, dtype=B3_DTYPE)
    return T, B1, B2, B3, xPrev, x, ism
