"""CPU restatement of the block list: structural properties and completeness.

The CUDA builder must reproduce these structures bit for bit (GPU tests); here
they are checked on their own terms: blocks are z-sorted column segments of at
most 32 atoms, the half-shell candidate set at rCut+pad contains every pair
within rCut exactly once, and exclusion masks cover every excluded pair.
"""
import numpy as np
import pytest

import oracle
from blade_b200 import systems


@pytest.fixture(scope="module", params=["water", "msld", "chain_small"])
def sysl(request):
    if request.param == "water":
        s = systems.water_box()
    elif request.param == "msld":
        s = systems.msld_water()
    else:
        s = systems.chain_in_water(seed=5, box=40.0, n_chain=600, n_wat=1800, rCut=12.0, rSwitch=10.0,
                                   name="chain_small")
    return s, oracle.build_list(s)


def test_domain_div_heuristic():
    # src/domdec/domdec.cu:114-117 evaluated for the two reference fixtures
    assert oracle.domain_div(648, [18.856] * 3) == (3, 3)
    assert oracle.domain_div(23558, [62.23] * 3) == (10, 10)


def test_blocks_partition_atoms(sysl):
    s, L = sysl
    B = L["blockCount"]
    bb = L["blockBounds"]
    assert bb[0] == 0 and bb[-1] == s.N
    assert (np.diff(bb) >= 1).all() and (np.diff(bb) <= 32).all()
    slot = L["slotAtom"].reshape(B, 32)
    atoms = slot[slot >= 0]
    assert np.array_equal(np.sort(atoms), np.arange(s.N))
    assert np.array_equal(L["sortedAtom"], slot[slot >= 0])


def test_columns_sorted_by_z(sysl):
    s, L = sysl
    xyz = s.xyz
    box = s.box
    divx, divy = L["divX"], L["divY"]
    w = xyz - np.floor(xyz / box) * box
    col = np.clip(np.floor(w[:, 0] / box[0] * divx).astype(int), 0, divx - 1) * divy + \
        np.clip(np.floor(w[:, 1] / box[1] * divy).astype(int), 0, divy - 1)
    srt = L["sortedAtom"]
    c = col[srt]
    assert (np.diff(c) >= 0).all()
    z = w[srt, 2]
    same = np.diff(c) == 0
    assert (np.diff(z)[same] >= 0).all()


def test_list_is_deterministic(sysl):
    s, L = sysl
    L2 = oracle.build_list(s)
    for k in ("blockBounds", "sortedAtom", "cand", "candExcl", "masks", "bmin", "bmax"):
        assert np.array_equal(L[k], L2[k])


def _pair_tiles(s, L):
    """Map every in-cutoff pair to its tile and check coverage and masks."""
    from scipy.spatial import cKDTree
    xyz = s.xyz.astype(np.float64)
    box = s.box.astype(np.float64)
    wrapped = np.mod(xyz, box)
    tree = cKDTree(wrapped, boxsize=box)
    pairs = tree.query_pairs(s.rCut, output_type="ndarray")
    B = L["blockCount"]
    slot_of = np.empty(s.N, np.int64)
    sl = L["slotAtom"]
    slot_of[sl[sl >= 0]] = np.nonzero(sl >= 0)[0]
    packed, bmin, bmax = oracle.pack(L, s.xyz, s.box)
    a, b = pairs[:, 0], pairs[:, 1]
    pa, pb = packed[slot_of[a]].astype(np.float64), packed[slot_of[b]].astype(np.float64)
    # image shift s such that pb + s*box is the minimum image of pa
    sh = np.round((pa - pb) / box).astype(int)
    return pairs, slot_of, sh


def test_every_pair_in_exactly_one_active_tile(sysl):
    s, L = sysl
    pairs, slot_of, sh = _pair_tiles(s, L)
    codes = {oracle.shift_vector(c): c for c in range(14)}
    tiles = {}
    for i in range(L["blockCount"]):
        for c in range(L["candStart"][i], L["candStart"][i + 1]):
            j, code = L["cand"][c]
            tiles[(i, int(j), int(code))] = c
    packed, bmin, bmax = oracle.pack(L, s.xyz, s.box)
    active = oracle.active_tiles(L, bmin, bmax, s.box, s.rCut)
    excl = set(map(tuple, s.excl.tolist()))
    missing = 0
    for (a, b), v in zip(pairs, sh):
        if (int(a), int(b)) in excl:
            continue
        ba, bb_ = slot_of[a] // 32, slot_of[b] // 32
        t = tuple(int(x) for x in v)
        if t in codes and not (t == (0, 0, 0) and bb_ < ba):
            key = (ba, bb_, codes[t])
        else:
            key = (bb_, ba, codes[tuple(-x for x in t)])
        c = tiles.get(key)
        if c is None or not active[c]:
            missing += 1
    assert missing == 0


def test_masks_cover_exclusions(sysl):
    s, L = sysl
    slot_of = np.empty(s.N, np.int64)
    sl = L["slotAtom"]
    slot_of[sl[sl >= 0]] = np.nonzero(sl >= 0)[0]
    lookup = {}
    for i in range(L["blockCount"]):
        for c in range(L["candStart"][i], L["candStart"][i + 1]):
            lookup.setdefault((i, int(L["cand"][c][0])), []).append(c)
    for a, b in s.excl[:2000]:
        ia, ib = slot_of[a], slot_of[b]
        for c in lookup.get((ia // 32, ib // 32), []):
            m = L["candExcl"][c]
            assert m >= 0
            assert not (L["masks"][m][ia % 32] >> (ib % 32)) & 1
