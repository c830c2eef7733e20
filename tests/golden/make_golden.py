"""Generates the golden vectors of tests/golden from the reference itself.

Runs the reference's own CUDA direct-space path (src/nbdirect + src/domdec,
unmodified, built into oracle/_ref/libbladeref.so by oracle/ref/Makefile) on
the seeded synthetic systems and stores coordinates, FP32 forces (dU/dx),
dU/dlambda and the nbdirect energy.  Needs a GPU:

    python tests/golden/make_golden.py OUTDIR [--pairs-only]

Cases: the 216-water box under all nine elecMethod x vdwMethod combinations,
the MSLD water box (soft core on and off), and the 23,558-atom chain-in-water
system (forces of the first 3,000 atoms kept); and, from the reference's
getforce_nb14 / getforce_nbex (src/bonded/pair.cu), pairs_*.npz for a small
chain-in-water system (1-4 pairs with e14fac 0.5 under three method
combinations, PME exclusion corrections) and the MSLD water box; and, from
the reference's getforce_ewald / getforce_ewaldself (src/nbrecip/nbrecip.cu),
pme_*.npz: reciprocal-space dU/dx, energy and dU/dlambda plus the self term
for the water box (orders 4, 6, 8), the MSLD water box and a small
chain-in-water system (--pme-only makes just these); and, from the
reference's holonomic_position / holonomic_velocity
(src/holonomic/holonomic.cu), holonomic_*.npz for rigid waters and
X-H groups of one to three hydrogens (--holonomic-only makes just these).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from blade_b200 import systems  # noqa: E402
from oracle import refgpu  # noqa: E402


def cases():
    for e in range(3):
        for v in range(3):
            s = systems.water_box()
            s.elecMethod, s.vdwMethod = e, v
            yield f"water216_e{e}v{v}", s, None
    yield "msld_water_soft", systems.msld_water(), None
    s = systems.msld_water()
    s.msld.useSoftCore = False
    yield "msld_water_hard", s, None
    yield "chain_water_23558", systems.chain_in_water(), 3000


def pair_cases():
    """(name, system, which, soft14, atoms kept) of the nb14 / nbex fixtures."""
    base = systems.chain_in_water(seed=5, box=30.0, n_chain=250, n_wat=780, name="chain_water_small")
    for e, v in ((1, 0), (0, 1), (2, 2)):
        s = systems.with_pair_lists(base, e14fac=0.5)
        s.elecMethod, s.vdwMethod = e, v
        yield f"pairs_nb14_e{e}v{v}", s, "nb14", False, 400
    s = systems.with_pair_lists(base, e14fac=0.5)
    yield "pairs_nbex", s, "nbex", False, None
    m = systems.with_pair_lists(systems.msld_water())
    yield "pairs_msld_nb14_soft", m, "nb14", True, None
    yield "pairs_msld_nb14_hard", m, "nb14", False, None
    yield "pairs_msld_nbex", m, "nbex", False, None


def pme_cases():
    """(name, system, order, grid) of the PME fixtures; grids from 1 A spacing."""
    from oracle import pme_oracle
    for order in (4, 6, 8):
        s = systems.water_box()
        yield f"pme_water216_o{order}", s, order, [pme_oracle.grid_size(L, 1.0) for L in s.box]
    s = systems.msld_water()
    yield "pme_msld_water", s, 6, [pme_oracle.grid_size(L, 1.0) for L in s.box]
    s = systems.chain_in_water(seed=5, box=30.0, n_chain=250, n_wat=780, name="chain_water_small")
    yield "pme_chain_small", s, 6, [pme_oracle.grid_size(L, 1.0) for L in s.box]


def holonomic_cases(out):
    from oracle import holonomic_oracle as H
    for name, jitter in (("holonomic_small_drift", 0.01), ("holonomic_large_drift", 0.05)):
        T, B1, B2, B3, xp, x, ism = H.test_clusters(seed=3, jitter=jitter)
        halfdt = 0.5 * 0.002 / 4.88882129e-02  # 2 fs in AKMA time units
        xr, vr = refgpu.holonomic("position", T, B1, B2, B3, xp, x, np.zeros_like(x), ism, halfdt, 1e-10)
        v_in = np.random.default_rng(4).normal(0, 5, x.shape)
        _, vv = refgpu.holonomic("velocity", T, B1, B2, B3, xp, xr, v_in, ism, halfdt, 1e-10)
        np.savez_compressed(os.path.join(out, name + ".npz"), x_prev=xp, x=x, ism=ism, halfdt=np.float64(halfdt),
                            tri=T.view(np.uint8), b1=B1.view(np.uint8), b2=B2.view(np.uint8), b3=B3.view(np.uint8),
                            x_ref=xr, v_ref=vr.astype(np.float32), v_in=v_in, v_proj_ref=vv.astype(np.float32))
        print(name, len(T), len(B1), len(B2), len(B3), flush=True)


def main(out, pairs_only=False, pme_only=False, holonomic_only=False):
    os.makedirs(out, exist_ok=True)
    if holonomic_only:
        holonomic_cases(out)
        return
    for name, s, order, K in pme_cases():
        ref = refgpu.RefGPU(s)
        ref.set_pme(order, K)
        r = ref.evaluate_pme("recip")
        r2 = ref.evaluate_pme("self")
        np.savez_compressed(os.path.join(out, name + ".npz"), xyz=s.xyz.astype(np.float32),
                            grad=r["grad"].astype(np.float32), energy=np.float64(r["energy"]),
                            lambdaForce=r["lambdaForce"].astype(np.float64),
                            self_energy=np.float64(r2["energy"]), self_lambdaForce=r2["lambdaForce"].astype(np.float64),
                            K=np.int64(K), order=np.int64(order), beta=np.float64(s.betaEwald))
        print(name, K, order, r["energy"], r2["energy"], flush=True)
    if pme_only:
        return
    for name, s, keep in ([] if pairs_only else cases()):
        r = refgpu.RefGPU(s).evaluate()
        g = r["grad"].astype(np.float32)
        n = s.N if keep is None else keep
        np.savez_compressed(os.path.join(out, name + ".npz"), xyz=s.xyz.astype(np.float32),
                            grad=g[:n], energy=np.float64(r["energy"]),
                            lambdaForce=r["lambdaForce"].astype(np.float64), n_forces=np.int64(n),
                            elecMethod=np.int64(s.elecMethod), vdwMethod=np.int64(s.vdwMethod))
        print(name, s.N, r["energy"], flush=True)
    for name, s, which, soft, keep in pair_cases():
        ref = refgpu.RefGPU(s)
        ref.set_pairs(soft)
        r = ref.evaluate_pairs(which)
        n = s.N if keep is None else keep
        np.savez_compressed(os.path.join(out, name + ".npz"), xyz=s.xyz.astype(np.float32),
                            grad=r["grad"].astype(np.float32)[:n], energy=np.float64(r["energy"]),
                            lambdaForce=r["lambdaForce"].astype(np.float64), n_forces=np.int64(n),
                            elecMethod=np.int64(s.elecMethod), vdwMethod=np.int64(s.vdwMethod))
        print(name, which, len(s.nb14), len(s.nbex), r["energy"], flush=True)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    main(args[0] if args else os.path.join(ROOT, "golden_out"), pairs_only="--pairs-only" in sys.argv,
         pme_only="--pme-only" in sys.argv, holonomic_only="--holonomic-only" in sys.argv)
