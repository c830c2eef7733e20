"""Seeded synthetic molecular systems for the nonbonded direct-space path.

No benchmark dataset exists for this path; these generators stand in for the
reference's own fixtures (``test/water216`` for the 216-water box and
``test/newDHFR`` for the 23,558-atom protein box) with the shapes, sizes and
parameter distributions of the workloads:

* ``water_box``     216 TIP3P waters on a 6x6x6 lattice, 18.856 A cube.
* ``chain_in_water`` a self-avoiding 1.5 A-bond chain solute plus TIP3P water
  filling the rest of a cubic box (62.23 A / 23,558 atoms by default).
* ``msld_water``    the water box plus MSLD perturbation sites
  (3 sites x 4 substituents of 8-15 atoms).
* ``batch_replicas`` uneven chain-in-water MSLD replicas, 3k-30k atoms.
* ``water_box_tric`` TIP3P waters in a triclinic cell (State::tricBox layout).
* ``load_fixture``  the reference's own water216 and newDHFR fixtures, as the
  golden-vector script stored them (tests/golden/fixture_*.npz).

Units are AKMA (A, kcal/mol, e).  Parameters follow the reference's tables:
TIP3P charges/LJ from ``test/toppar_water_ions/par_water_ions.prm:77-78``,
LJ pair table c12 = eps*Rmin^12, c6 = 2*eps*Rmin^6 with eps = sqrt(eps_i eps_j)
and Rmin = Rmin/2_i + Rmin/2_j (``src/system/potential.cxx:1393-1403``),
exclusion lists with both orders of every pair (``potential.cxx:1156-1163``),
MSLD ``siteBlock = (site<<16)|block`` (``src/msld/msld.cu:470-476``) and
mutual exclusion of substituents at one site (``potential.cxx:1035-1050``).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

KELEC_AKMA = 332.0716          # src/main/defines.h:55
SOFTCORE_RADIUS_AKMA = 4.0     # src/main/defines.h:48

TIP3P_Q_O, TIP3P_Q_H = -0.834, 0.417
TIP3P_EPS_O, TIP3P_RH_O = 0.1521, 1.7682
TIP3P_EPS_H, TIP3P_RH_H = 0.046, 0.2245
TIP3P_ROH, TIP3P_THETA = 0.9572, math.radians(104.52)

NBOND_DTYPE = np.dtype([("siteBlock", "<i4"), ("q", "<f4"), ("typeIdx", "<i4")])
# Same layouts as struct Nb14Potential / NbExPotential, src/system/potential.h:91-104.
NB14_DTYPE = np.dtype([("idx", "<i4", 2), ("siteBlock", "<i4", 2), ("qxq", "<f4"), ("c12", "<f4"), ("c6", "<f4"),
                       ("e14fac", "<f4")])
NBEX_DTYPE = np.dtype([("idx", "<i4", 2), ("siteBlock", "<i4", 2), ("qxq", "<f4")])


@dataclasses.dataclass
class Msld:
    """MSLD block layout: block 0 is the environment (site 0)."""
    blockCount: int
    siteCount: int
    siteBound: np.ndarray        # [siteCount+1] int32
    lambdaSite: np.ndarray       # [blockCount] int32
    theta: np.ndarray            # [blockCount] float64
    fnex: float = 5.5            # src/msld/msld.cu:48
    useSoftCore: bool = True


@dataclasses.dataclass
class System:
    name: str
    xyz: np.ndarray              # [N,3] float32
    box: np.ndarray              # [3] float32 (orthorhombic edges)
    nbonds: np.ndarray           # [N] NBOND_DTYPE
    vdw: np.ndarray              # [T,T,2] float32 (c12, c6)
    excl: np.ndarray             # [E,2] int32 directed pairs (both orders)
    rCut: float
    rSwitch: float
    betaEwald: float
    elecMethod: int = 1          # PME
    vdwMethod: int = 0           # VFSWITCH
    msld: Msld | None = None
    cullPad: float = 2.0
    nb14: np.ndarray | None = None       # NB14_DTYPE 1-4 pairs (with_pair_lists)
    nbex: np.ndarray | None = None       # NBEX_DTYPE excluded pairs for the PME correction
    bonds: np.ndarray | None = None      # [B,2] int32 covalent bonds (one order), for dynamics only
    bond_param: np.ndarray | None = None  # [B,2] float32 (kb, b0): U = kb/2 (r - b0)^2
    masses: np.ndarray | None = None      # [N] amu, when the system comes with its own
    tric: np.ndarray | None = None        # [3] (B_x, C_x, C_y) of a triclinic cell, else None

    def box6(self) -> np.ndarray:
        """(A_x, B_y, C_z, B_x, C_x, C_y): box edges, then the off-diagonal
        components of the lower-triangular cell (zero when orthorhombic)."""
        t = np.zeros(3, np.float32) if self.tric is None else np.asarray(self.tric, np.float32)
        return np.concatenate([np.asarray(self.box, np.float32), t]).astype(np.float32)

    def tric_box(self) -> np.ndarray:
        """The cell in the layout of State::tricBox_f: A_x, B_x, B_y, C_x, C_y, C_z."""
        b = self.box6()
        return np.array([b[0], b[3], b[1], b[4], b[5], b[2]], np.float32)

    @property
    def N(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def nTypes(self) -> int:
        return int(self.vdw.shape[0])

    def lambdas(self) -> np.ndarray:
        """lambda per block from theta (FP64), block 0 fixed at 1."""
        if self.msld is None:
            return np.ones(1)
        m = self.msld
        lam = np.ones(m.blockCount)
        for s in range(1, m.siteCount):
            a, b = m.siteBound[s], m.siteBound[s + 1]
            e = np.exp(m.fnex * np.sin(m.theta[a:b]))
            lam[a:b] = e / e.sum()
        return lam


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def vdw_table(eps: np.ndarray, rhalf: np.ndarray) -> np.ndarray:
    """Pair table in FP32 following potential.cxx:1393-1403."""
    eps = np.asarray(eps, np.float32)
    rh = np.asarray(rhalf, np.float32)
    e = np.sqrt(eps[:, None] * eps[None, :]).astype(np.float32)
    s = (rh[:, None] + rh[None, :]).astype(np.float32)
    s6 = (s * s).astype(np.float32)
    s6 = (s6 * (s6 * s6)).astype(np.float32)
    t = np.empty(e.shape + (2,), np.float32)
    t[..., 0] = (e * s6 * s6).astype(np.float32)
    t[..., 1] = (np.float32(2) * e * s6).astype(np.float32)
    return t


def random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices (quaternion method)."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def tip3p_local() -> np.ndarray:
    h = TIP3P_THETA / 2
    return np.array([[0, 0, 0],
                     [TIP3P_ROH * math.sin(h), 0, TIP3P_ROH * math.cos(h)],
                     [-TIP3P_ROH * math.sin(h), 0, TIP3P_ROH * math.cos(h)]])


def place_waters(rng, sites: np.ndarray, jitter: float) -> np.ndarray:
    rot = random_rotations(rng, len(sites))
    loc = tip3p_local()
    o = sites + rng.uniform(-jitter, jitter, size=sites.shape)
    return (o[:, None, :] + np.einsum("nij,aj->nai", rot, loc)).reshape(-1, 3)


def water_excl(first_atom: int, nwat: int) -> np.ndarray:
    base = first_atom + 3 * np.arange(nwat)
    pairs = []
    for a, b in ((0, 1), (0, 2), (1, 2)):
        pairs.append(np.stack([base + a, base + b], 1))
        pairs.append(np.stack([base + b, base + a], 1))
    return np.concatenate(pairs).astype(np.int32)


def chain_walk(rng, n: int, center: np.ndarray, radius: float, bond: float = 1.5,
               dmin: float = 2.2, start: np.ndarray | None = None,
               avoid: np.ndarray | None = None) -> np.ndarray:
    """Self-avoiding walk of n atoms, 1.5 A bonds, confined to a sphere.

    Non-bonded atoms (|i-j|>2) stay >= dmin apart; ``avoid`` holds atoms the
    walk must also keep dmin away from.  A walk that jams is restarted in a
    sphere 12 % wider (up to six times).
    """
    for _ in range(6):
        try:
            return _chain_walk_once(rng, n, center, radius, bond, dmin, start, avoid)
        except RuntimeError:
            radius *= 1.12
    raise RuntimeError("chain_walk: could not place chain")


def _chain_walk_once(rng, n, center, radius, bond, dmin, start, avoid) -> np.ndarray:
    """One attempt: each step proposes 24 directions at once and checks them
    against a dense cell grid; dead ends backtrack."""
    K, SLOTS = 24, 8
    start = np.asarray(center if start is None else start, np.float64)
    lo = np.minimum(start, center) - radius - 2 * dmin
    span = 2 * radius + 4 * dmin + np.abs(start - center)
    dims = np.maximum(1, np.ceil(span / dmin).astype(int)) + 1
    grid = np.full((*dims, SLOTS), -1, np.int64)
    fill = np.zeros(tuple(dims), np.int64)
    navoid = 0 if avoid is None else len(avoid)
    allpos = np.zeros((n + navoid, 3))           # avoid atoms stored after the chain
    offs = np.array([(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)])

    def cell_of(p):
        return np.clip(np.floor((p - lo) / dmin).astype(int), 0, dims - 1)

    def insert(idx, p):
        c = tuple(cell_of(p))
        k = fill[c]
        if k < SLOTS:
            grid[c + (k,)] = idx
            fill[c] = k + 1

    def remove(idx, p):
        c = tuple(cell_of(p))
        row = grid[c]
        k = int(np.nonzero(row == idx)[0][0])
        row[k:-1] = row[k + 1:].copy()
        row[-1] = -1
        fill[c] -= 1

    for a in range(navoid):
        allpos[n + a] = avoid[a]
        insert(n + a, avoid[a])
    allpos[0] = start
    insert(0, start)
    i, fails = 1, 0
    r2max, dmin2 = radius * radius, dmin * dmin
    while i < n:
        v = rng.normal(size=(K, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        if i >= 2:
            prev = allpos[i - 1] - allpos[i - 2]
            prev /= np.linalg.norm(prev)
            dot = v @ prev
            back = dot < -0.3                     # no sharp back-turns (angle > ~107 deg)
            v[back] -= 1.3 * dot[back, None] * prev
            v /= np.linalg.norm(v, axis=1, keepdims=True)
        p = allpos[i - 1] + bond * v
        good = ((p - center) ** 2).sum(1) <= r2max
        cells = np.clip(np.floor((p - lo) / dmin).astype(int)[:, None, :] + offs[None], 0, dims - 1)
        nb = grid[cells[..., 0], cells[..., 1], cells[..., 2]].reshape(K, -1)   # [K, 27*SLOTS]
        valid = (nb >= 0) & ~((nb < n) & (nb >= i - 2))
        q = allpos[np.maximum(nb, 0)]
        d2 = ((q - p[:, None, :]) ** 2).sum(-1)
        clash = (valid & (d2 < dmin2)).any(1)
        cand = np.nonzero(good & ~clash)[0]
        if len(cand):
            allpos[i] = p[cand[0]]
            insert(i, allpos[i])
            i += 1
            continue
        fails += 1
        if fails > 20000:
            raise RuntimeError("chain_walk: could not place chain")
        for _ in range(min(i - 1, 1 + int(rng.integers(0, 4)))):
            i -= 1
            remove(i, allpos[i])
    return allpos[:n].copy()


# Bond force constants of the dynamics stand-in for bonded terms and SHAKE
# (kb of U = kb/2 (r-b0)^2, kcal/mol/A^2): TIP3P O-H and H-H, backbone bonds.
KB_OH, KB_HH, KB_CHAIN = 900.0, 200.0, 600.0


def chain_bonds(first: int, n: int) -> np.ndarray:
    a = first + np.arange(n - 1)
    return np.stack([a, a + 1], 1).astype(np.int32)


def water_bonds(first: int, nwat: int) -> tuple[np.ndarray, np.ndarray]:
    """O-H1, O-H2, H1-H2 of each water and their force constants."""
    o = first + 3 * np.arange(nwat)
    b = np.concatenate([np.stack([o, o + 1], 1), np.stack([o, o + 2], 1), np.stack([o + 1, o + 2], 1)])
    kb = np.repeat([KB_OH, KB_OH, KB_HH], nwat)
    return b.astype(np.int32), kb


def with_bond_lengths(xyz: np.ndarray, bonds: np.ndarray, kb: np.ndarray) -> np.ndarray:
    """(kb, b0) per bond with b0 the bond's length in ``xyz``."""
    b0 = np.linalg.norm(xyz[bonds[:, 0]].astype(np.float64) - xyz[bonds[:, 1]], axis=1)
    return np.stack([kb, b0], 1).astype(np.float32)


def bond_csr(N: int, bonds: np.ndarray, param: np.ndarray):
    """Per-atom bond lists (both ends of every bond), stable in bond order."""
    b = np.concatenate([bonds, bonds[:, ::-1]]).astype(np.int64)
    prm = np.concatenate([param, param]).astype(np.float32)
    order = np.argsort(b[:, 0], kind="stable")
    start = np.zeros(N + 1, np.int64)
    np.add.at(start, b[:, 0] + 1, 1)
    return np.cumsum(start).astype(np.int32), b[order, 1].astype(np.int32), np.ascontiguousarray(prm[order])


def chain_excl(first: int, n: int) -> np.ndarray:
    pairs = []
    for d in (1, 2):
        a = first + np.arange(n - d)
        pairs.append(np.stack([a, a + d], 1))
        pairs.append(np.stack([a + d, a], 1))
    return np.concatenate(pairs).astype(np.int32) if pairs else np.zeros((0, 2), np.int32)


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def water_box(seed: int = 1, n_side: int = 6, box: float = 18.856, jitter: float = 0.3,
              rCut: float = 9.0, rSwitch: float = 8.0, beta: float = 0.34) -> System:
    """216 TIP3P waters, 6x6x6 lattice, seeded orientations, +-0.3 A jitter."""
    rng = np.random.default_rng(seed)
    a = box / n_side
    g = (np.arange(n_side) + 0.5) * a
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    xyz = place_waters(rng, sites, jitter).astype(np.float32)
    nw = len(sites)
    nb = np.zeros(3 * nw, NBOND_DTYPE)
    nb["q"] = np.tile(np.float32([TIP3P_Q_O, TIP3P_Q_H, TIP3P_Q_H]), nw)
    # type 0 = HT (most frequent), type 1 = OT, like the count-sorted type list
    nb["typeIdx"] = np.tile(np.int32([1, 0, 0]), nw)
    vdw = vdw_table([TIP3P_EPS_H, TIP3P_EPS_O], [TIP3P_RH_H, TIP3P_RH_O])
    return System("water216", xyz, np.float32([box] * 3), nb, vdw, water_excl(0, nw),
                  rCut, rSwitch, beta)


def water_box_tric(seed: int = 6, cell=(24.0, 7.0, 23.0, -6.0, 8.0, 22.5), n=(8, 8, 7), jitter: float = 0.3,
                   rCut: float = 9.0, rSwitch: float = 8.0, beta: float = 0.34) -> System:
    """TIP3P waters on a lattice spanning a triclinic cell, given in the layout
    of State::tricBox_f (A_x, B_x, B_y, C_x, C_y, C_z): A = (A_x,0,0),
    B = (B_x,B_y,0), C = (C_x,C_y,C_z).  Sites at fractional coordinates
    ((i+1/2)/n0, (j+1/2)/n1, (k+1/2)/n2), seeded orientations and jitter;
    coordinates are left unwrapped (inside the parallelepiped, not the brick)."""
    rng = np.random.default_rng(seed)
    ax, bx, by, cx, cy, cz = (float(v) for v in cell)
    A, B, C = np.array([ax, 0, 0]), np.array([bx, by, 0]), np.array([cx, cy, cz])
    f = [(np.arange(k) + 0.5) / k for k in n]
    u = np.stack(np.meshgrid(*f, indexing="ij"), -1).reshape(-1, 3)
    sites = u[:, :1] * A + u[:, 1:2] * B + u[:, 2:3] * C
    xyz = place_waters(rng, sites, jitter).astype(np.float32)
    nw = len(sites)
    nb = np.zeros(3 * nw, NBOND_DTYPE)
    nb["q"] = np.tile(np.float32([TIP3P_Q_O, TIP3P_Q_H, TIP3P_Q_H]), nw)
    nb["typeIdx"] = np.tile(np.int32([1, 0, 0]), nw)
    vdw = vdw_table([TIP3P_EPS_H, TIP3P_EPS_O], [TIP3P_RH_H, TIP3P_RH_O])
    s = System("water_tric", xyz, np.float32([ax, by, cz]), nb, vdw, water_excl(0, nw), rCut, rSwitch, beta)
    s.tric = np.float32([bx, cx, cy])
    return s


def _fill_water(rng, box: float, nwat: int, solute: np.ndarray, dmin: float = 2.6):
    from scipy.spatial import cKDTree
    n_side = max(2, int(round(box / (1 / 0.0334) ** (1 / 3))))
    while True:
        a = box / n_side
        g = (np.arange(n_side) + 0.5) * a
        sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
        if len(solute):
            tree = cKDTree(np.mod(solute, box), boxsize=box)
            d, _ = tree.query(np.mod(sites, box), k=1)
            sites = sites[d > dmin]
        if len(sites) >= nwat:
            break
        n_side += 1
    pick = np.sort(rng.choice(len(sites), nwat, replace=False))
    return place_waters(rng, sites[pick], 0.3)


def _lj_types(rng, n: int):
    eps = rng.uniform(0.02, 0.2, n).astype(np.float32)
    rh = rng.uniform(1.2, 2.1, n).astype(np.float32)
    return eps, rh


def chain_in_water(seed: int = 2, box: float = 62.23, n_chain: int = 2489, n_wat: int = 7023,
                   rCut: float = 12.0, rSwitch: float = 10.0, beta: float = 0.32,
                   name: str = "chain_water_23558") -> System:
    """Protein-sized system: self-avoiding chain solute + TIP3P water, ~23.5k atoms.

    Chain atoms carry per-atom LJ parameters drawn from U(0.02,0.2) kcal/mol
    and U(1.2,2.1) A, i.e. one LJ type per chain atom.
    """
    rng = np.random.default_rng(seed)
    center = np.full(3, box / 2)
    radius = (3 * n_chain / (4 * math.pi * 0.06)) ** (1 / 3)
    chain = chain_walk(rng, n_chain, center, radius)
    q = rng.normal(0, 0.35, n_chain)
    q -= q.mean()
    wat = _fill_water(rng, box, n_wat, chain)
    xyz = np.concatenate([chain, wat]).astype(np.float32)
    N = len(xyz)
    nb = np.zeros(N, NBOND_DTYPE)
    nb["q"][:n_chain] = q.astype(np.float32)
    nb["q"][n_chain:] = np.tile(np.float32([TIP3P_Q_O, TIP3P_Q_H, TIP3P_Q_H]), n_wat)
    eps_c, rh_c = _lj_types(rng, n_chain)
    # types: 0 HT, 1 OT, 2.. chain atoms
    eps = np.concatenate([[TIP3P_EPS_H, TIP3P_EPS_O], eps_c])
    rh = np.concatenate([[TIP3P_RH_H, TIP3P_RH_O], rh_c])
    nb["typeIdx"][:n_chain] = 2 + np.arange(n_chain)
    nb["typeIdx"][n_chain:] = np.tile(np.int32([1, 0, 0]), n_wat)
    excl = np.concatenate([chain_excl(0, n_chain), water_excl(n_chain, n_wat)])
    return System(name, xyz, np.float32([box] * 3), nb, vdw_table(eps, rh), excl,
                  rCut, rSwitch, beta)


def _nearby(points: np.ndarray | None, center: np.ndarray, cut: float, box: float) -> np.ndarray | None:
    """Minimum images of ``points`` within ``cut`` of ``center``."""
    if points is None or len(points) == 0:
        return None
    d = points - center
    d -= box * np.round(d / box)
    keep = (d * d).sum(1) < cut * cut
    return center + d[keep] if keep.any() else None


def _add_sites(rng, fixed_atoms, anchors: np.ndarray, subs_per_site, box: float, dmin: float = 2.2,
               avoid_sites: bool = True, outward: np.ndarray | None = None, shared_geometry: bool = False):
    """Grow substituents at each anchor; returns atoms, per-atom (site, block), exclusions.

    Substituents of one site overlap each other (they are alternatives and
    mutually excluded); they keep ``dmin`` from ``fixed_atoms`` (the solute)
    and, with ``avoid_sites``, from the substituents of the other sites, with
    which they interact.  ``outward`` (unit vectors, one per site) moves the
    walks' sphere 4 A off the anchor, away from the solute.  With
    ``shared_geometry`` the substituents of a site share one walk of 8-15
    atoms (alchemical variants of one shape, differing in charges and LJ
    types) instead of independent walks.
    """
    atoms, site_block, bonds_excl, site_members = [], [], [], []
    block = 1
    offset = 0
    other = np.zeros((0, 3))
    for s, (anc, nsub) in enumerate(zip(anchors, subs_per_site), start=1):
        members = []
        site_atoms = []
        # with an outward direction, the walks' sphere sits beside the anchor
        out = None if outward is None else outward[s - 1]
        center = anc if out is None else anc + 4.0 * out
        near = [_nearby(fixed_atoms, center, 16.0, box)] + ([_nearby(other, center, 16.0, box)] if avoid_sites else [])
        near = [a for a in near if a is not None]
        avoid = np.concatenate(near) if near else None
        template = None
        for _ in range(nsub):
            n = int(rng.integers(8, 16)) if template is None or not shared_geometry else len(template)
            if template is None or not shared_geometry:
                start = anc + rng.normal(0, 0.3, 3) if out is None else anc + 2.0 * out + rng.normal(0, 0.3, 3)
                for t in range(200):                       # a start point clear of the avoided atoms
                    if avoid is None or ((avoid - start) ** 2).sum(1).min() >= dmin * dmin:
                        break
                    start = center + rng.normal(0, 0.6 + 0.02 * t, 3)
                template = chain_walk(rng, n, center, 6.0, start=start, avoid=avoid)
            walk = template
            site_atoms.append(walk)
            idx = offset + np.arange(n)
            atoms.append(walk)
            site_block += [(s, block)] * n
            bonds_excl.append(chain_excl(offset, n))
            members.append(idx)
            offset += n
            block += 1
        site_members.append(members)
        other = np.concatenate([other] + site_atoms)
    mut = []
    for members in site_members:
        for a in range(len(members)):
            for b in range(a + 1, len(members)):
                ia, ib = np.meshgrid(members[a], members[b], indexing="ij")
                p = np.stack([ia.ravel(), ib.ravel()], 1)
                mut += [p, p[:, ::-1]]
    excl = np.concatenate(bonds_excl + mut).astype(np.int32)
    return np.concatenate(atoms), site_block, excl, block


def _msld_layout(rng, subs_per_site, theta_range=(-math.pi / 2, math.pi / 2)) -> Msld:
    nb = 1 + int(sum(subs_per_site))
    bound = np.zeros(len(subs_per_site) + 2, np.int32)
    bound[1] = 1
    for i, k in enumerate(subs_per_site):
        bound[i + 2] = bound[i + 1] + k
    site = np.zeros(nb, np.int32)
    for s in range(1, len(bound) - 1):
        site[bound[s]:bound[s + 1]] = s
    theta = np.zeros(nb)
    theta[1:] = rng.uniform(*theta_range, nb - 1)
    return Msld(nb, len(bound) - 1, bound, site, theta)


def msld_water(seed: int = 3, sites: int = 3, subs: int = 4, clear: float = 2.2,
               avoid_sites: bool = False, charge_sigma: float = 0.35, rigid_substituents: bool = False,
               shared_geometry: bool = False, variant_sigma: float | None = None, variant_lj_atoms: int = 3,
               tie_variants: bool = False) -> System:
    """MSLD water box: the 216-water box plus MSLD sites anchored on water O's.

    Waters with any atom within ``clear`` A of a substituent are removed.
    ``avoid_sites`` keeps substituents of different sites 2.2 A apart (for
    dynamics; off by default so the seeded parity systems stay as they are).
    ``charge_sigma`` is the spread of substituent charges (e).
    ``rigid_substituents`` excludes every pair inside one substituent (a rigid
    fragment: its internal energy does not change with lambda);
    ``shared_geometry`` makes the substituents of a site variants of one shape;
    with ``variant_sigma`` (needs ``shared_geometry``) they are also variants of
    one fragment's parameters: the first substituent's charges plus
    N(0, variant_sigma) e and its LJ types with ``variant_lj_atoms`` atoms
    changed (eps x U(0.8,1.25), Rmin/2 x U(0.92,1.08)), as R-groups that
    differ at a few atoms.  ``tie_variants`` (needs
    ``shared_geometry``) adds zero-length bonds from every atom of a site's
    first substituent to the same atom of the others, so that substituents
    out of play (lambda ~ 0, hardly any nonbonded force) stay in place instead
    of drifting through the solvent, as the unscaled bonded terms to the
    common core hold them in a real MSLD system.
    """
    base = water_box(seed)
    rng = np.random.default_rng(seed + 1000)
    nw = base.N // 3
    L = float(base.box[0])
    while True:  # anchors at least 9 A apart (minimum image) so sites do not overlap
        anchor_w = rng.choice(nw, sites, replace=False)
        anchors = base.xyz[3 * anchor_w].astype(np.float64)
        d = anchors[:, None, :] - anchors[None, :, :]
        d -= L * np.round(d / L)
        dd = np.sqrt((d ** 2).sum(-1)) + 1e9 * np.eye(sites)
        if dd.min() >= 9.0:
            break
    subs_xyz, sb, sub_excl, nblock = _add_sites(rng, None, anchors, [subs] * sites, float(base.box[0]),
                                                avoid_sites=avoid_sites, shared_geometry=shared_geometry)
    from scipy.spatial import cKDTree
    tree = cKDTree(np.mod(subs_xyz, base.box[0]), boxsize=float(base.box[0]))
    d, _ = tree.query(np.mod(base.xyz.astype(np.float64), base.box[0]), k=1)
    bad = (d < clear).reshape(nw, 3).any(1)
    keep = np.nonzero(~bad)[0]
    wat = base.xyz.reshape(nw, 3, 3)[keep].reshape(-1, 3)
    ns = len(subs_xyz)
    xyz = np.concatenate([subs_xyz, wat]).astype(np.float32)
    N = len(xyz)
    nbd = np.zeros(N, NBOND_DTYPE)
    q = rng.normal(0, charge_sigma, ns)
    # each substituent neutral
    sbs = np.array(sb)
    for blk in np.unique(sbs[:, 1]):
        m = sbs[:, 1] == blk
        q[m] -= q[m].mean()
    nbd["q"][:ns] = q.astype(np.float32)
    nbd["siteBlock"][:ns] = (sbs[:, 0] << 16) | sbs[:, 1]
    nbd["q"][ns:] = np.tile(np.float32([TIP3P_Q_O, TIP3P_Q_H, TIP3P_Q_H]), len(keep))
    eps_s, rh_s = _lj_types(rng, ns)
    if variant_sigma is not None and shared_geometry:
        first = {}
        for blk in np.unique(sbs[:, 1]):
            m = np.nonzero(sbs[:, 1] == blk)[0]
            site = int(sbs[m[0], 0])
            if site not in first:
                first[site] = m
                continue
            b0 = first[site]
            dq = rng.normal(0, variant_sigma, len(m))
            q[m] = q[b0] + dq - dq.mean()
            eps_s[m], rh_s[m] = eps_s[b0], rh_s[b0]
            redo = m[rng.choice(len(m), min(variant_lj_atoms, len(m)), replace=False)]
            eps_s[redo] *= rng.uniform(0.8, 1.25, len(redo)).astype(np.float32)
            rh_s[redo] *= rng.uniform(0.92, 1.08, len(redo)).astype(np.float32)
        nbd["q"][:ns] = q.astype(np.float32)
    eps = np.concatenate([[TIP3P_EPS_H, TIP3P_EPS_O], eps_s])
    rh = np.concatenate([[TIP3P_RH_H, TIP3P_RH_O], rh_s])
    nbd["typeIdx"][:ns] = 2 + np.arange(ns)
    nbd["typeIdx"][ns:] = np.tile(np.int32([1, 0, 0]), len(keep))
    excl = np.concatenate([sub_excl, water_excl(ns, len(keep))])
    sizes = np.bincount(sbs[:, 1])[1:]
    if rigid_substituents:
        intra = []
        for f, n in zip(np.concatenate([[0], np.cumsum(sizes)[:-1]]), sizes):
            a, b = np.meshgrid(np.arange(f, f + n), np.arange(f, f + n), indexing="ij")
            keep_ab = a != b
            intra.append(np.stack([a[keep_ab], b[keep_ab]], 1))
        excl = np.unique(np.concatenate([excl] + intra).astype(np.int32), axis=0)
    msld = _msld_layout(rng, [subs] * sites)
    firsts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    wb, wkb = water_bonds(ns, len(keep))
    ties = []
    if tie_variants and shared_geometry:
        site_first = {}
        for f, n, blk in zip(firsts, sizes, range(1, len(sizes) + 1)):
            site = int(sbs[f, 0])
            if site not in site_first:
                site_first[site] = f
            else:
                f0 = site_first[site]
                ties.append(np.stack([f0 + np.arange(n), f + np.arange(n)], 1))
    bonds = np.concatenate([chain_bonds(f, n) for f, n in zip(firsts, sizes)] + ties + [wb]).astype(np.int32)
    kb = np.concatenate([np.full(len(bonds) - len(wb), KB_CHAIN), wkb])
    return System(f"msld_water_{N}", xyz, base.box.copy(), nbd, vdw_table(eps, rh), excl,
                  base.rCut, base.rSwitch, base.betaEwald, msld=msld, bonds=bonds,
                  bond_param=with_bond_lengths(xyz, bonds, kb))


MSLD_CHAIN_DENSITY = 0.0965   # atoms per A^3 of the msld_chain replicas


def msld_chain(seed: int, n_atoms: int, n_sites: int, subs_per_site, rCut=12.0, rSwitch=10.0,
               beta=0.32) -> System:
    """MSLD replica: chain solute + water + MSLD sites on chain atoms, density 0.0965 A^-3."""
    rng = np.random.default_rng(seed)
    box = (n_atoms / MSLD_CHAIN_DENSITY) ** (1 / 3)
    n_chain = max(60, int(0.1 * n_atoms))
    center = np.full(3, box / 2)
    radius = (3 * n_chain / (4 * math.pi * 0.06)) ** (1 / 3)
    chain = chain_walk(rng, n_chain, center, radius)
    # sites on surface atoms of the chain globule, grown outward into the water
    rad = np.linalg.norm(chain - chain.mean(0), axis=1)
    surface = np.arange(5, n_chain - 5)
    surface = surface[rad[surface] >= np.quantile(rad[surface], 0.8)]
    anchors_idx = rng.choice(surface, n_sites, replace=False)
    anchors = chain[anchors_idx]
    outward = anchors - chain.mean(0)
    outward /= np.linalg.norm(outward, axis=1, keepdims=True)
    subs_xyz, sb, sub_excl, nblock = _add_sites(rng, chain, anchors, subs_per_site, box, outward=outward)
    solute = np.concatenate([chain, subs_xyz])
    ns = len(subs_xyz)
    n_wat = max(0, (n_atoms - len(solute)) // 3)
    wat = _fill_water(rng, box, n_wat, solute)
    xyz = np.concatenate([subs_xyz, chain, wat]).astype(np.float32)
    N = len(xyz)
    nbd = np.zeros(N, NBOND_DTYPE)
    q = rng.normal(0, 0.35, ns + n_chain)
    sbs = np.array(sb)
    for blk in np.unique(sbs[:, 1]):
        m = np.nonzero(sbs[:, 1] == blk)[0]
        q[m] -= q[m].mean()
    q[ns:] -= q[ns:].mean()
    nbd["q"][:ns + n_chain] = q.astype(np.float32)
    nbd["siteBlock"][:ns] = (sbs[:, 0] << 16) | sbs[:, 1]
    nbd["q"][ns + n_chain:] = np.tile(np.float32([TIP3P_Q_O, TIP3P_Q_H, TIP3P_Q_H]), n_wat)
    eps_s, rh_s = _lj_types(rng, ns + n_chain)
    eps = np.concatenate([[TIP3P_EPS_H, TIP3P_EPS_O], eps_s])
    rh = np.concatenate([[TIP3P_RH_H, TIP3P_RH_O], rh_s])
    nbd["typeIdx"][:ns + n_chain] = 2 + np.arange(ns + n_chain)
    nbd["typeIdx"][ns + n_chain:] = np.tile(np.int32([1, 0, 0]), n_wat)
    excl = np.concatenate([sub_excl, chain_excl(ns, n_chain), water_excl(ns + n_chain, n_wat)])
    msld = _msld_layout(rng, list(subs_per_site))
    sizes = np.bincount(sbs[:, 1])[1:]
    firsts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    wb, wkb = water_bonds(ns + n_chain, n_wat)
    bonds = np.concatenate([chain_bonds(f, n) for f, n in zip(firsts, sizes)] + [chain_bonds(ns, n_chain), wb])
    kb = np.concatenate([np.full(len(bonds) - len(wb), KB_CHAIN), wkb])
    return System(f"msld_chain_{N}", xyz, np.float32([box] * 3), nbd, vdw_table(eps, rh), excl,
                  rCut, rSwitch, beta, msld=msld, bonds=bonds, bond_param=with_bond_lengths(xyz, bonds, kb))


def batch_replicas(n_rep: int = 64, seed: int = 4, n_min: int = 3000, n_max: int = 30000):
    """Uneven MSLD replicas: sizes log-uniform in [3k, 30k], 1-3 sites x 2-5 substituents."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(n_rep):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        ns = int(rng.integers(1, 4))
        subs = [int(k) for k in rng.integers(2, 6, ns)]
        out.append(msld_chain(seed * 1000 + r, n, ns, subs))
    return out


def excl_csr(N: int, excl: np.ndarray):
    """Per-atom sorted exclusion partners (CSR)."""
    if len(excl) == 0:
        return np.zeros(N + 1, np.int32), np.zeros(0, np.int32)
    e = np.unique(excl.astype(np.int64), axis=0)
    e = e[e[:, 0] != e[:, 1]]
    order = np.lexsort((e[:, 1], e[:, 0]))
    e = e[order]
    start = np.zeros(N + 1, np.int64)
    np.add.at(start, e[:, 0] + 1, 1)
    return np.cumsum(start).astype(np.int32), e[:, 1].astype(np.int32)


def _pair_site_blocks(a: int, b: int):
    """(siteBlock[0], siteBlock[1]) of a pair as the pair kernel reads them
    (src/bonded/pair.cu:224-231): the perturbed block first, the second slot
    only for two blocks of different sites; None for two blocks of one site
    (mutually excluded, never present together)."""
    if a == b:
        return (a, 0)
    if a == 0 or b == 0:
        return (a or b, 0)
    if (a >> 16) == (b >> 16):
        return None
    return (a, b)


def with_pair_lists(s: System, e14fac: float = 1.0) -> System:
    """Copy of ``s`` with 1-4 pair lists (Potential::nb14s, src/system/potential.cxx:1093-1140)
    and PME exclusion-correction lists (Potential::nbexs, potential.cxx:1144-1160).

    1-4 pairs are (i, i+3) along runs of consecutive bonded atoms of one block
    ((i,i+1), (i+1,i+2), (i+2,i+3) all excluded); they join the exclusions of
    the direct space and get c12/c6 from the LJ table and the given e14fac.
    The correction list holds every other excluded pair i<j.
    """
    import dataclasses as dc
    ex = set(map(tuple, np.asarray(s.excl).tolist()))
    sb = s.nbonds["siteBlock"]
    q = s.nbonds["q"].astype(np.float64)
    t = s.nbonds["typeIdx"]
    p14 = []
    for i in range(s.N - 3):
        if all((i + k, i + k + 1) in ex for k in range(3)) and len({int(sb[i + k]) for k in range(4)}) == 1:
            p14.append((i, i + 3))
    nb14 = np.zeros(len(p14), NB14_DTYPE)
    for n, (i, j) in enumerate(p14):
        nb14[n]["idx"] = (i, j)
        nb14[n]["siteBlock"] = _pair_site_blocks(int(sb[i]), int(sb[j]))
        nb14[n]["qxq"] = np.float32(q[i] * q[j])
        nb14[n]["c12"], nb14[n]["c6"] = s.vdw[t[i], t[j]]
        nb14[n]["e14fac"] = e14fac
    excl = np.asarray(s.excl)
    if p14:
        a = np.array(p14, np.int32)
        excl = np.unique(np.concatenate([excl, a, a[:, ::-1]]), axis=0)
    s14 = set(p14)
    rows = []
    for i, j in excl.tolist():
        if i < j and (i, j) not in s14:
            blocks = _pair_site_blocks(int(sb[i]), int(sb[j]))
            if blocks is not None:
                rows.append(((i, j), blocks, np.float32(q[i] * q[j])))
    nbex = np.zeros(len(rows), NBEX_DTYPE)
    for n, (ij, blocks, qq) in enumerate(rows):
        nbex[n]["idx"], nbex[n]["siteBlock"], nbex[n]["qxq"] = ij, blocks, qq
    return dc.replace(s, name=s.name + "_pairs", excl=excl.astype(np.int32), nb14=nb14, nbex=nbex)



def load_fixture(path: str) -> System:
    """A System stored by the golden-vector script from one of the reference's
    own CHARMM fixtures (test/water216, test/newDHFR): coordinates, box,
    charges, LJ type indices and table, exclusions (each pair once, i < j;
    both orders are restored here, as potential.cxx:1156-1163 lists them),
    1-4 and exclusion-correction lists in the reference's layouts, bonds and
    masses, and the cutoffs the fixture is evaluated with."""
    z = np.load(path)
    N = len(z["q"])
    nb = np.zeros(N, NBOND_DTYPE)
    nb["q"] = z["q"]
    nb["typeIdx"] = z["typeIdx"]
    half = z["excl_half"].astype(np.int32)
    excl = np.concatenate([half, half[:, ::-1]])
    excl = excl[np.lexsort((excl[:, 1], excl[:, 0]))]
    s = System(str(z["name"]), z["xyz"].astype(np.float32), z["box"].astype(np.float32), nb,
               z["vdw"].astype(np.float32), excl, float(z["rCut"]), float(z["rSwitch"]), float(z["beta"]))
    s.nb14 = z["nb14"].view(NB14_DTYPE).copy()
    s.nbex = z["nbex"].view(NBEX_DTYPE).copy()
    s.bonds = z["bonds"].astype(np.int32)
    s.masses = z["masses"].astype(np.float64)
    return s
