"""GPU parity: libbnb (through the C ABI) against the FP64 oracle.

Tolerances: force RMS error relative to the oracle's RMS force <= 1e-5 (the
path's accuracy target); dU/dlambda likewise; energy within 1e-5 relative to
max(|E|, N kcal/mol); in-cutoff pair counts exact; list structures bit-exact.
"""
import numpy as np
import pytest
import torch

import oracle
from blade_b200 import systems
from blade_b200.nbdirect import NbDirect

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def rel_rms(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def run(sys_, count=True):
    nb = NbDirect(sys_)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    nb.set_counting(count)
    f, l, e = nb.evaluate(pos)
    torch.cuda.synchronize()
    out = {"grad": f.cpu().numpy(), "lambdaForce": l.cpu().numpy(), "energy": float(e[0]),
           "pairs": nb.pair_count() if count else None, "status": nb.status()}
    nb.close()
    return out


def check(sys_, g, o, check_lambda=False):
    assert g["status"] == 0
    # FP32 vs FP64 distance: pairs within ~1e-6 A of rCut may flip (about one
    # pair per 4e6 at rCut 12 A); the list itself misses nothing (bit-exact
    # list tests and the oracle coverage test).
    assert abs(g["pairs"] - o["pairs"]) <= max(2, 1e-6 * o["pairs"]), (g["pairs"], o["pairs"])
    err = rel_rms(g["grad"], o["grad"])
    assert err <= FORCE_TOL, err
    scale = max(abs(o["energy"]), sys_.N)
    assert abs(g["energy"] - o["energy"]) <= 1e-5 * scale, (g["energy"], o["energy"])
    if check_lambda:
        lerr = rel_rms(g["lambdaForce"][1:], o["lambdaForce"][1:])
        assert lerr <= FORCE_TOL, lerr
    return err


def test_water216_parity(cuda):
    s = systems.water_box()
    check(s, run(s), oracle.nbdirect(s))


def test_chain_water_23558_parity(cuda):
    s = systems.chain_in_water()
    assert s.N == 23558
    check(s, run(s), oracle.nbdirect(s))


def test_msld_parity(cuda):
    s = systems.msld_water()
    check(s, run(s), oracle.nbdirect(s), check_lambda=True)


def test_msld_without_softcore(cuda):
    s = systems.msld_water()
    s.msld.useSoftCore = False
    check(s, run(s), oracle.nbdirect(s), check_lambda=True)


@pytest.mark.parametrize("elec,vdw", [(e, v) for e in range(3) for v in range(3)])
def test_all_methods(cuda, elec, vdw):
    s = systems.water_box()
    s.elecMethod, s.vdwMethod = elec, vdw
    check(s, run(s), oracle.nbdirect(s))


def test_msld_replica_combine_mode(cuda):
    """A 3k-atom MSLD replica: per-atom LJ types (combination mode) + soft core."""
    s = systems.msld_chain(11, 3000, 2, [3, 4])
    assert s.nTypes > 64
    check(s, run(s), oracle.nbdirect(s), check_lambda=True)


def test_unwrapped_coordinates(cuda):
    """Coordinates several box lengths outside the box give the same physics."""
    s = systems.water_box()
    s2 = systems.water_box()
    s2.xyz = (s.xyz + np.float32([3, -2, 5]) * s.box).astype(np.float32)
    check(s2, run(s2), oracle.nbdirect(s2))


def _wide_exclusions():
    """Water box whose first 8 atoms are each excluded with 40 atoms spread
    over the box: their blocks list more than 16 exclusion-partner blocks, so
    the builder's per-block partner list overflows and takes the full scan."""
    s = systems.water_box()
    rng = np.random.default_rng(8)
    extra = []
    for a in range(8):
        for b in rng.choice(np.arange(8, s.N), 40, replace=False):
            extra += [(a, int(b)), (int(b), a)]
    s.excl = np.unique(np.concatenate([s.excl, np.int32(extra)]), axis=0).astype(np.int32)
    s.name = "water_wide_excl"
    return s


def test_list_bitexact_against_oracle(cuda):
    for s in (systems.water_box(), systems.msld_water(), _wide_exclusions(),
              systems.chain_in_water(seed=5, box=40.0, n_chain=600, n_wat=1800, name="chain_small")):
        nb = NbDirect(s)
        pos = nb.positions_tensor()
        nb.update_domdec(pos, True)
        g = nb.get_list()
        o = oracle.build_list(s)
        for k in ("wrap", "blockBounds", "sortedAtom", "slotAtom", "bmin", "bmax", "candStart", "cand",
                  "candExcl", "masks"):
            assert np.array_equal(g[k], o[k]), (s.name, k)
        nb.close()


def test_deterministic_bits(cuda):
    s = systems.chain_in_water(seed=5, box=40.0, n_chain=600, n_wat=1800, name="chain_small")
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    a = nb.evaluate(pos)
    b = nb.evaluate(pos)
    nb.update_domdec(pos, True)
    c = nb.evaluate(pos)
    for x, y in ((a, b), (a, c)):
        assert torch.equal(x[0], y[0]) and torch.equal(x[2], y[2])
    nb.close()


def test_batch_equals_single_bitwise(cuda):
    """Replicas stepped in one launch give the same bits as one-at-a-time."""
    reps = [systems.msld_chain(20 + k, n, 1 + k % 2, [2 + k % 3] * (1 + k % 2)) for k, n in
            enumerate((3000, 3600, 4200))]
    nb = NbDirect(reps)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    fb, lb, eb = nb.evaluate(pos)
    for r, s in enumerate(reps):
        one = NbDirect(s)
        p1 = one.positions_tensor()
        one.update_domdec(p1, True)
        f1, l1, e1 = one.evaluate(p1)
        a0, a1 = nb.starts[r], nb.starts[r + 1]
        l0, l1_ = nb.lam_starts[r], nb.lam_starts[r + 1]
        assert torch.equal(fb[a0:a1], f1)
        assert torch.equal(lb[l0:l1_], l1)
        assert torch.equal(eb[r:r + 1], e1)
        one.close()
    nb.close()


def test_accumulates_into_reference_buffers(cuda):
    """force/lambdaForce/energy are ADDED (State::force_d semantics)."""
    s = systems.msld_water()
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    lam = nb.lambdas_tensor()
    force = torch.ones(3 * s.N, device="cuda")
    lf = torch.full((nb.L,), 2.0, device="cuda")
    en = torch.full((1,), 5.0, dtype=torch.float64, device="cuda")
    f64 = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
    nb.getforce_nbdirect(pos, lam, True, force=force, lambda_force=lf, energy=en, force64=f64)
    o = oracle.nbdirect(s)
    assert rel_rms(force.cpu().numpy() - 1.0, o["grad"].ravel()) <= 2e-5
    assert rel_rms(lf.cpu().numpy()[1:] - 2.0, o["lambdaForce"][1:]) <= 2e-5
    assert abs(float(en[0]) - 5.0 - o["energy"]) <= 1e-5 * max(abs(o["energy"]), s.N)
    nb.close()
