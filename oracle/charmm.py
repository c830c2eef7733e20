"""CHARMM PSF / CRD / parameter-file readers and the nonbonded tables the
reference builds from them (test infrastructure only: the golden-vector
script imports it to turn the reference's own fixtures -- test/water216 and
test/newDHFR -- into arrays; the arrays, not these files, travel with the
tests).

Restated from the reference:
* parameter files: Parameters::add_parameter_file / add_parameter_nbonds /
  add_parameter_nbfixs (src/system/parameters.cxx:129-160, 392-480): the
  NONBONDED section's lines `type ignored eps Rmin/2 [ignored eps14
  Rmin/2_14]`, eps stored as -eps (KCAL_MOL = 1 in CHARMM units), e14fac and
  GEOM from the continuation line, NBFIX lines `type1 type2 eps Rmin
  [eps14 Rmin14]`; tokens after '!' are comments; a line whose first four
  letters are a section keyword ends the section;
* PSF: Structure::add_structure_psf_file (src/system/structure.cxx:570-640):
  atoms (type name, charge, mass) and the bond list;
* CRD: Coordinates::file_crd (src/system/coordinates.cxx:209-275), atoms
  matched by segment, residue number and atom name;
* Potential::initialize (src/system/potential.cxx:930-1163, 1309-1420):
  exclusions as closures of the bond graph (1-2, then 1-3 from bonds x
  1-2 partners, then 1-4 from bonds x 1-3 partners), both orders of every
  pair; the 1-4 pair list with e14fac = sqrt(e14fac_i e14fac_j) and the
  eps14/Rmin14 parameters; the PME exclusion-correction list of the other
  excluded pairs; LJ types numbered by descending atom count (ties by name);
  the T x T table c12 = eps Rmin^12, c6 = 2 eps Rmin^6 with eps =
  sqrt(eps_i eps_j), Rmin = Rmin/2_i + Rmin/2_j (2 sqrt(..) when both types
  are GEOM), NBFIX pairs taken as given -- all in FP32 like the reference's
  `real`.
"""
from __future__ import annotations

import os

import numpy as np

SECTION_KEYS = ("ATOM", "BOND", "ANGL", "DIHE", "IMPR", "CMAP", "NONB", "NBFI", "HBON", "END")
NB_HEADER = ("NONBONDED", "CUTNB", "CTOFNB", "CTONNB", "EPS", "E14FAC", "WMIN", "GEOM")


def _tokens(line):
    out = []
    for t in line.split():
        if t.startswith("!"):
            break
        out.append(t)
    return out


def _float(tok, default=None):
    try:
        return float(tok)
    except (TypeError, ValueError):
        if default is None:
            raise
        return default


def read_parameters(paths):
    """nonbonded {type: (eps, rmin_half, eps14, rmin_half14, e14fac, geom)}
    and nbfix {(t1, t2): (eps, rmin, eps14, rmin14)} (keys in both orders),
    eps with the sign the reference stores (positive well depth)."""
    nb, fix = {}, {}
    for path in paths:
        with open(path) as f:
            lines = f.readlines()
        section = None
        e14fac, geom = 1.0, 0
        for raw in lines:
            if raw.startswith("*"):
                continue
            tok = _tokens(raw)
            if not tok:
                continue
            head = tok[0]
            up = head.upper()
            if section in ("NONB", "NBFI") and head[:4] not in SECTION_KEYS and up not in NB_HEADER:
                if section == "NONB":
                    eps = _float(tok[2])
                    rh = _float(tok[3])
                    eps14 = _float(tok[5] if len(tok) > 5 else None, eps)
                    rh14 = _float(tok[6] if len(tok) > 6 else None, rh)
                    nb[head] = (np.float32(-eps), np.float32(rh), np.float32(-eps14), np.float32(rh14),
                                np.float32(e14fac), geom)
                else:
                    eps, rm = _float(tok[2]), _float(tok[3])
                    eps14 = _float(tok[4] if len(tok) > 4 else None, eps)
                    rm14 = _float(tok[5] if len(tok) > 5 else None, rm)
                    v = (np.float32(-eps), np.float32(rm), np.float32(-eps14), np.float32(rm14))
                    fix[(head, tok[1])] = v
                    fix[(tok[1], head)] = v
                continue
            if section == "NONB" and up in NB_HEADER and up != "NONBONDED":
                for k, t in enumerate(tok):
                    if t.upper() == "E14FAC":
                        e14fac = float(tok[k + 1])
                    elif t.upper() == "GEOM":
                        geom = 1
                continue
            if head == "END":
                section = None
                continue
            key = head[:4]
            if key in SECTION_KEYS:
                section = key
                if key == "NONB":
                    e14fac, geom = 1.0, 0
    return nb, fix


def read_psf(path):
    """atoms: dict of arrays (seg, res, name, type, charge, mass); bonds
    [B,2] int (0-based, PSF order)."""
    with open(path) as f:
        lines = f.readlines()
    k = 0
    while "!NATOM" not in lines[k]:
        k += 1
    n = int(lines[k].split()[0])
    rows = [lines[k + 1 + i].split() for i in range(n)]
    atoms = {"seg": [r[1] for r in rows], "res": [r[2] for r in rows], "resname": [r[3] for r in rows],
             "name": [r[4] for r in rows], "type": [r[5] for r in rows],
             "charge": np.array([float(r[6]) for r in rows], np.float32),
             "mass": np.array([float(r[7]) for r in rows], np.float64)}
    k += 1 + n
    while "!NBOND" not in lines[k]:
        k += 1
    nbond = int(lines[k].split()[0])
    vals = []
    k += 1
    while len(vals) < 2 * nbond:
        vals.extend(int(t) for t in lines[k].split())
        k += 1
    bonds = np.array(vals, np.int64).reshape(-1, 2) - 1
    return atoms, bonds


def read_crd(path, atoms):
    """[N,3] float64 coordinates in PSF atom order."""
    with open(path) as f:
        lines = [l for l in f.readlines() if not l.startswith("*")]
    n = int(lines[0].split()[0])
    pos = {}
    for l in lines[1:1 + n]:
        t = l.split()
        pos[(t[7], t[8], t[3])] = (float(t[4]), float(t[5]), float(t[6]))
    return np.array([pos[(s, r, a)] for s, r, a in zip(atoms["seg"], atoms["res"], atoms["name"])], np.float64)


def exclusion_sets(N, bonds):
    """(allExcl, bondExcl, angleExcl, diheExcl) as lists of sets, built in the
    reference's order (potential.cxx:967-1030, no virtual sites or MSLD)."""
    allx = [set() for _ in range(N)]
    b12 = [set() for _ in range(N)]
    b13 = [set() for _ in range(N)]
    b14 = [set() for _ in range(N)]
    for i, j in bonds:
        for a, b in ((i, j), (j, i)):
            if b not in allx[a]:
                b12[a].add(b)
                allx[a].add(b)
    for src, dst in ((b12, b13), (b13, b14)):
        for i, j in bonds:
            for a, c in ((i, j), (j, i)):
                for k in sorted(src[c]):      # partners of the other bond end
                    if k == a:
                        continue
                    for p, q in ((a, k), (k, a)):
                        if q not in allx[p]:
                            dst[p].add(q)
                            allx[p].add(q)
    return allx, b12, b13, b14


def _combine(np_i, np_j, fourteen=False):
    eps_i, rh_i = (np_i[2], np_i[3]) if fourteen else (np_i[0], np_i[1])
    eps_j, rh_j = (np_j[2], np_j[3]) if fourteen else (np_j[0], np_j[1])
    eps = np.float32(np.sqrt(np.float32(eps_i * eps_j)))
    if np_i[5] == 1 and np_j[5] == 1:
        sig = np.float32(2 * np.sqrt(np.float32(rh_i * rh_j)))
    else:
        sig = np.float32(rh_i + rh_j)
    return eps, sig


def _c12c6(eps, sig):
    s6 = np.float32(sig * sig)
    s6 = np.float32(s6 * np.float32(s6 * s6))
    return np.float32(np.float32(eps * s6) * s6), np.float32(2 * np.float32(eps * s6))


def build(psf, crd, params, box, rCut, rSwitch, beta, name, elecMethod=1, vdwMethod=0):
    """A blade_b200.systems.System of the fixture, with its 1-4 and PME
    exclusion-correction lists, covalent bonds and masses."""
    from blade_b200 import systems
    atoms, bonds = read_psf(psf)
    xyz = read_crd(crd, atoms)
    nbp, fix = read_parameters(params)
    N = len(atoms["type"])
    types = atoms["type"]
    count = {}
    for t in types:
        count[t] = count.get(t, 0) + 1
    order = sorted(count, key=lambda t: (-count[t], t))
    lookup = {t: i for i, t in enumerate(order)}
    T = len(order)
    vdw = np.zeros((T, T, 2), np.float32)
    for i, ti in enumerate(order):
        for j, tj in enumerate(order):
            if (ti, tj) in fix:
                eps, sig = fix[(ti, tj)][0], fix[(ti, tj)][1]
            else:
                eps, sig = _combine(nbp[ti], nbp[tj])
            vdw[i, j] = _c12c6(eps, sig)
    nb = np.zeros(N, systems.NBOND_DTYPE)
    nb["q"] = atoms["charge"]
    nb["typeIdx"] = [lookup[t] for t in types]
    allx, _, _, b14 = exclusion_sets(N, bonds)
    excl = np.array([(i, j) for i in range(N) for j in sorted(allx[i])], np.int32).reshape(-1, 2)
    nb14 = []
    for i in range(N):
        for j in sorted(b14[i]):
            if i < j:
                ti, tj = types[i], types[j]
                e14 = np.float32(np.sqrt(nbp[ti][4]) * np.sqrt(nbp[tj][4]))
                if (ti, tj) in fix:
                    eps, sig = fix[(ti, tj)][2], fix[(ti, tj)][3]
                else:
                    eps, sig = _combine(nbp[ti], nbp[tj], fourteen=True)
                c12, c6 = _c12c6(eps, sig)
                nb14.append(((i, j), (0, 0), np.float32(atoms["charge"][i] * atoms["charge"][j]), c12, c6, e14))
    nbex = []
    for i in range(N):
        for j in sorted(allx[i]):
            if i < j and j not in b14[i]:
                nbex.append(((i, j), (0, 0), np.float32(atoms["charge"][i] * atoms["charge"][j])))
    s = systems.System(name, xyz.astype(np.float32), np.float32(box), nb, vdw, excl, rCut, rSwitch, beta,
                       elecMethod=elecMethod, vdwMethod=vdwMethod)
    s.nb14 = np.array(nb14, systems.NB14_DTYPE)
    s.nbex = np.array(nbex, systems.NBEX_DTYPE)
    s.bonds = bonds.astype(np.int32)
    s.masses = atoms["mass"]
    return s


def save_fixture(s, path):
    """Stores ``s`` in the layout blade_b200.systems.load_fixture reads."""
    half = s.excl[s.excl[:, 0] < s.excl[:, 1]]
    np.savez_compressed(path, name=np.str_(s.name), xyz=s.xyz.astype(np.float32), box=np.float32(s.box),
                        q=s.nbonds["q"].astype(np.float32), typeIdx=s.nbonds["typeIdx"].astype(np.int16),
                        vdw=s.vdw.astype(np.float32), excl_half=half.astype(np.int32),
                        nb14=s.nb14.view(np.uint8), nbex=s.nbex.view(np.uint8), bonds=s.bonds.astype(np.int32),
                        masses=s.masses.astype(np.float32), rCut=np.float64(s.rCut), rSwitch=np.float64(s.rSwitch),
                        beta=np.float64(s.betaEwald))


def fixture_paths(reference_root):
    """(psf, crd, parameter files, box) of the reference's own fixtures."""
    t = os.path.join(reference_root, "test")
    return {
        "water216": (os.path.join(t, "water216", "minimized.psf"), os.path.join(t, "water216", "minimized.crd"),
                     [os.path.join(t, "toppar", "par_all36_prot.prm"),
                      os.path.join(t, "toppar_water_ions", "par_water_ions.prm")], [18.856] * 3),
        "dhfr": (os.path.join(t, "newDHFR", "5dfr.psf"), os.path.join(t, "newDHFR", "5dfr.crd"),
                 [os.path.join(t, "newDHFR", "par_all22_prot.inp")], [62.23] * 3),
    }
