"""Randomised parity sweep on the GPU: seeded systems of four kinds (water
box, chain in water, MSLD water box with or without soft core, triclinic
water cell) with random electrostatics x van der Waals methods, cutoffs and
tunings (tiles per work item, CTAs per SM, work-list tail), each against the
FP64 oracle.  Every system is evaluated twice on one list -- the first launch
takes its work items in list order, the second in the longest-first order
the first one measured -- and the two must agree bit for bit."""
import numpy as np
import pytest
import torch

import oracle
from blade_b200 import systems
from blade_b200.nbdirect import NbDirect

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5    # relative RMS of dU/dx and dU/dlambda against FP64
ENERGY_TOL = 1e-5   # per max(|E|, N)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def _system(seed):
    rng = np.random.default_rng(1000 + seed)
    kind = seed % 4
    if kind == 0:
        n = int(rng.integers(6, 8))
        s = systems.water_box(seed=seed, n_side=n, box=18.856 * n / 6, rCut=float(rng.choice([8.0, 9.0])),
                              rSwitch=7.0)
    elif kind == 1:
        box = float(rng.uniform(30.0, 38.0))
        s = systems.chain_in_water(seed=seed, box=box, n_chain=int(rng.integers(150, 500)),
                                   n_wat=int(0.0334 * box ** 3 * 0.8), rCut=float(rng.choice([9.0, 10.0, 12.0])),
                                   rSwitch=8.0, name=f"chain_sweep_{seed}")
    elif kind == 2:
        s = systems.msld_water(seed=seed)
        s.msld.useSoftCore = bool(rng.integers(0, 2))
    else:
        s = systems.water_box_tric(seed=seed)
    s.elecMethod, s.vdwMethod = int(rng.integers(0, 3)), int(rng.integers(0, 3))
    tuning = (int(rng.choice([1, 2, 4, 8, 16, 32])), int(rng.choice([0, 2, 3])), int(rng.choice([0, 2])))
    return s, tuning


@pytest.mark.parametrize("seed", range(12))
def test_random_system_matches_oracle_in_both_orders(cuda, seed):
    s, tuning = _system(seed)
    nb = NbDirect(s)
    nb.set_tuning(*tuning)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    nb.set_counting(True)
    first = nb.evaluate(pos)                 # items in list order; measures their cycles
    pairs = nb.pair_count()
    second = nb.evaluate(pos)                # items longest first
    torch.cuda.synchronize()
    assert nb.status() == 0
    for x, y in zip(first, second):
        assert torch.equal(x, y), (s.name, tuning)
    o = oracle.nbdirect(s)
    g = first[0].cpu().numpy()
    assert _rel(g, o["grad"]) <= FORCE_TOL, (s.name, s.elecMethod, s.vdwMethod, tuning)
    e = float(first[2][0])
    assert abs(e - o["energy"]) <= ENERGY_TOL * max(abs(o["energy"]), s.N), (e, o["energy"])
    assert abs(pairs - o["pairs"]) <= max(2, 1e-6 * o["pairs"]), (pairs, o["pairs"])
    if s.msld is not None:
        lf = first[1].cpu().numpy()
        assert _rel(lf[1:], o["lambdaForce"][1:]) <= FORCE_TOL
    nb.close()
