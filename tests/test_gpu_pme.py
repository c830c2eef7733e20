"""PME reciprocal space and Ewald self term on the GPU (bnb_compute_pme /
bnb_compute_ewald_self) against the FP64 oracle restatement
(oracle/pme_oracle.py) and the reference's own getforce_ewald /
getforce_ewaldself golden vectors: interpolation orders 4, 6 and 8, MSLD
scaling, several replicas with their own grids on one handle, unwrapped
coordinates, repeated calls and the grid rule."""
import glob
import os

import numpy as np
import pytest
import torch

from blade_b200 import systems
from blade_b200.nbdirect import NbDirect
from oracle import pme_oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FORCE_TOL = 2e-5      # relative RMS of dU/dx vs FP64 (FP32 B-splines and FFT, fixed-point grid)
ENERGY_TOL = 1e-5
DUDL_TOL = 2e-5
REF_FORCE_TOL = 1e-4  # against the reference's FP32 build (fast math, FP32 atomics)
K_ELECTRIC = 332.0716


def _rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def _oracle(s, order, K, xyz=None):
    lam = s.lambdas() if s.msld else None
    sb = s.nbonds["siteBlock"]
    return pme_oracle.pme_recip(s.xyz if xyz is None else xyz, s.nbonds["q"], s.box, K, order, s.betaEwald,
                                K_ELECTRIC, sb, lam)


def _small_chain():
    return systems.chain_in_water(seed=5, box=30.0, n_chain=250, n_wat=780, name="chain_water_small")


@pytest.mark.parametrize("order", [4, 6, 8])
def test_recip_matches_oracle(cuda, order):
    s = systems.water_box()
    nb = NbDirect(s)
    nb.set_pme(order=order, grid_space=1.0)
    K = nb.pme_grid(0)
    assert K == tuple(pme_oracle.grid_size(L, 1.0) for L in s.box)
    f, _, e = nb.evaluate_pme()
    E, g, _, _ = _oracle(s, order, K)
    assert _rel(f.cpu().numpy(), g) < FORCE_TOL
    assert float(e.cpu()[0]) == pytest.approx(E, rel=ENERGY_TOL)
    nb.close()


def test_msld_recip_and_self(cuda):
    s = systems.msld_water()
    nb = NbDirect(s)
    nb.set_pme(order=6)
    K = nb.pme_grid(0)
    f, l, e = nb.evaluate_pme()
    E, g, lf, _ = _oracle(s, 6, K)
    assert _rel(f.cpu().numpy(), g) < FORCE_TOL
    assert float(e.cpu()[0]) == pytest.approx(E, rel=ENERGY_TOL)
    assert _rel(l.cpu().numpy()[1:], lf[1:]) < DUDL_TOL
    ls, es = nb.evaluate_ewald_self()
    Es, lfs = pme_oracle.ewald_self(s.nbonds["q"], s.betaEwald, K_ELECTRIC, s.nbonds["siteBlock"], s.lambdas())
    assert float(es.cpu()[0]) == pytest.approx(Es, rel=1e-6)
    assert _rel(ls.cpu().numpy()[1:], lfs[1:]) < 1e-6
    nb.close()


def test_repeat_is_bitwise(cuda):
    s = _small_chain()
    nb = NbDirect(s)
    nb.set_pme(order=6)
    a = nb.evaluate_pme()
    b = nb.evaluate_pme()
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    nb.close()


def test_replicas_match_single_handles(cuda):
    """Three replicas (two share a grid size: one batched FFT plan) on one
    handle agree with three one-replica handles.  The batched cuFFT plan may
    round differently from the single one, so the comparison is to FP32
    rounding, not bitwise; each handle on its own is bitwise repeatable."""
    reps = [systems.water_box(), systems.water_box(seed=7), systems.water_box(seed=9, n_side=8, box=25.14)]
    nb = NbDirect(reps)
    nb.set_pme(order=6)
    f, l, e = nb.evaluate_pme()
    f = f.cpu().numpy()
    off = 0
    for r, s in enumerate(reps):
        one = NbDirect(s)
        one.set_pme(order=6)
        assert one.pme_grid(0) == nb.pme_grid(r)
        f1, _, e1 = one.evaluate_pme()
        assert _rel(f[off:off + s.N], f1.cpu().numpy()) < 1e-6
        assert float(e[r].cpu()) == pytest.approx(float(e1[0].cpu()), rel=1e-7)
        off += s.N
        one.close()
    nb.close()


def test_unwrapped_coordinates(cuda):
    s = systems.water_box()
    nb = NbDirect(s)
    nb.set_pme(order=6)
    K = nb.pme_grid(0)
    x2 = (s.xyz + np.float32([3, -2, 5]) * s.box).astype(np.float32)
    f, _, e = nb.evaluate_pme(positions=nb.positions_tensor([x2]))
    E, g, _, _ = _oracle(s, 6, K)
    assert _rel(f.cpu().numpy(), g) < FORCE_TOL
    assert float(e.cpu()[0]) == pytest.approx(E, rel=ENERGY_TOL)
    nb.close()


def test_explicit_grid_and_accumulating_outputs(cuda):
    s = systems.water_box()
    nb = NbDirect(s)
    nb.set_pme(order=6, grid=(24, 20, 27))
    assert nb.pme_grid(0) == (24, 20, 27)
    pos = nb.positions_tensor()
    force = torch.full((3 * s.N,), 1.0, dtype=torch.float32, device="cuda")
    energy = torch.full((1,), 2.0, dtype=torch.float64, device="cuda")
    nb.getforce_ewald(pos, None, True, force=force, energy=energy)
    E, g, _, _ = _oracle(s, 6, (24, 20, 27))
    assert _rel(force.cpu().numpy().reshape(-1, 3) - 1.0, g) < 1e-4
    assert float(energy.cpu()[0]) - 2.0 == pytest.approx(E, rel=ENERGY_TOL)
    nb.close()


GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "pme_*.npz")))


def _golden_case(name):
    if name.startswith("pme_msld"):
        return systems.msld_water()
    if name.startswith("pme_chain"):
        return _small_chain()
    return systems.water_box()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(f)[:-4] for f in GOLDEN])
def test_recip_matches_reference_golden(cuda, path):
    z = np.load(path)
    s = _golden_case(os.path.basename(path)[:-4])
    assert np.array_equal(s.xyz, z["xyz"])
    nb = NbDirect(s)
    nb.set_pme(order=int(z["order"]), grid=tuple(int(k) for k in z["K"]))
    f, l, e = nb.evaluate_pme()
    assert _rel(f.cpu().numpy(), z["grad"]) < REF_FORCE_TOL
    assert float(e.cpu()[0]) == pytest.approx(float(z["energy"]), rel=1e-4)
    ls, es = nb.evaluate_ewald_self()
    assert float(es.cpu()[0]) == pytest.approx(float(z["self_energy"]), rel=1e-5)
    if s.msld:
        assert _rel(l.cpu().numpy()[1:], z["lambdaForce"][1:]) < REF_FORCE_TOL
        assert _rel(ls.cpu().numpy()[1:], z["self_lambdaForce"][1:]) < 1e-5
    nb.close()


def test_zero_charges_and_non_pme_methods(cuda):
    s = systems.water_box()
    s.nbonds["q"] = 0
    nb = NbDirect(s)
    nb.set_pme(order=6)
    f, _, e = nb.evaluate_pme()
    assert float(f.abs().max().cpu()) == 0.0 and float(e.cpu()[0]) == 0.0
    ls, es = nb.evaluate_ewald_self()
    assert float(es.cpu()[0]) == 0.0
    nb.close()
    s2 = systems.water_box()
    s2.elecMethod = 0                                # FSWITCH: no reciprocal space (nbrecip.cu:486)
    nb = NbDirect(s2)
    nb.set_pme(order=6)
    e64 = torch.full((1,), 5.0, dtype=torch.float64, device="cuda")
    f64 = torch.full((3 * s2.N,), 7.0, dtype=torch.float64, device="cuda")
    nb.getforce_ewald(nb.positions_tensor(), None, True, force64=f64, energy64=e64)
    nb.getforce_ewaldself(None, True, energy64=e64)
    torch.cuda.synchronize()
    assert float(e64.cpu()[0]) == 5.0 and bool((f64 == 7.0).all())
    nb.close()


def test_capture_in_cuda_graph(cuda):
    """The reciprocal evaluation (cuFFT plans made beforehand) records into a
    CUDA graph; replays give the eager bits."""
    s = systems.water_box()
    nb = NbDirect(s)
    nb.set_pme(order=6)
    pos = nb.positions_tensor()
    f_eager, _, e_eager = nb.evaluate_pme(pos)
    f64 = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
    e64 = torch.zeros(1, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):                       # warm-up outside capture
        nb.getforce_ewald(pos, None, True, force64=f64, energy64=e64)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        nb.getforce_ewald(pos, None, True, force64=f64, energy64=e64)
    f64.zero_()
    e64.zero_()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(f64.reshape(-1, 3), f_eager) and torch.equal(e64, e_eager)
    del g
    nb.close()


def test_total_electrostatics_matches_oracle_and_is_beta_invariant(cuda):
    """The four electrostatic pieces on the GPU -- bnb_compute (direct),
    bnb_compute_nbex, bnb_compute_pme, bnb_compute_ewald_self -- add up to
    the oracle's Ewald total, and the total does not depend on beta."""
    import dataclasses as dc
    import oracle
    base = systems.with_pair_lists(systems.water_box())
    q = base.nbonds["q"].astype(np.float64)
    totals = []
    for beta in (0.34, 0.40):
        s = dc.replace(base, betaEwald=beta)
        nb = NbDirect(s)
        pos = nb.positions_tensor()
        nb.update_domdec(pos, True)
        ed = float(nb.evaluate(pos)[2][0])
        nb.set_pairs()
        ex = float(nb.evaluate_pairs("nbex", pos)[2][0])
        nb.set_pme(order=8, grid=(40, 40, 40))
        er = float(nb.evaluate_pme(pos)[2][0])
        es = float(nb.evaluate_ewald_self()[1][0])
        nb.close()
        parts = (oracle.nbdirect(s)["energy"], oracle.pair_lists(s, which="nbex")["energy"],
                 pme_oracle.pme_recip(s.xyz, q, s.box, [40, 40, 40], 8, beta, K_ELECTRIC)[0],
                 pme_oracle.ewald_self(q, beta, K_ELECTRIC)[0])
        scale = max(abs(p) for p in parts)
        assert abs((ed + ex + er + es) - sum(parts)) < 2e-6 * scale
        totals.append(ed + ex + er + es)
    assert abs(totals[0] - totals[1]) < 2e-5 * scale
