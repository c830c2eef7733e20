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
X-H groups of one to three hydrogens (--holonomic-only makes just these);
and, from the reference's Msld::calc_lambda_from_theta,
calc_thetaForce_from_lambdaForce, getforce_fixedBias / getforce_variableBias
(src/msld/msld.cu:863-1153) and State::update (src/update/update.cu:233-305),
msld_maps*.npz and update_msld_water.npz (--msld-only makes just these);
and the reference's own CHARMM fixtures: `make_golden.py REFERENCE_ROOT
--fixtures` (CPU) turns test/water216 and test/newDHFR into
fixture_<name>.npz, and `--real-only` (GPU) evaluates the reference's direct
space, nb14, nbex, PME and self terms on them into real_<name>.npz; and the
reference's triclinic direct space on triclinic water boxes, tric_*.npz
(--tric-only), and its triclinic PME reciprocal space on them,
tric_pme_*.npz (--tric-pme-only).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
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


MSLD_BOUND = np.array([0, 1, 5, 9, 13], np.int32)          # environment + 3 sites x 4 substituents
MSLD_SITE = np.repeat(np.arange(4), np.diff(MSLD_BOUND)).astype(np.int32)


def msld_varbias(rng):
    """Every variable-bias type the reference evaluates (1-12) on pairs of
    substituents of one site and across sites, parameters in their usual
    ranges (k in kcal/mol; l0 the soft-core offset or the exponent)."""
    from blade_b200.msld import VARBIAS_DTYPE
    spec = [(6, 0.0, 0), (8, 0.017, 0), (10, -5.56, 0), (1, 0.8, 2), (2, 0.2, 2), (3, 0.0, 2), (4, 0.5, 0),
            (5, 0.0, 0), (7, 0.1, 0), (9, 0.5, 3), (11, 2.0, 2), (12, 0.1, 2), (1, 0.8, 3), (3, 0.0, 3)]
    vb = np.zeros(len(spec) * 2, VARBIAS_DTYPE)
    for k, (t, l0, n) in enumerate(spec):
        for r in range(2):
            a = 1 + rng.integers(0, 12)
            b = 1 + rng.integers(0, 12)
            while b == a:
                b = 1 + rng.integers(0, 12)
            vb[2 * k + r] = (a, b, t, l0, rng.uniform(-4, 4), n)
    return vb


def msld_cases(out):
    """Msld::calc_lambda_from_theta, calc_thetaForce_from_lambdaForce and the
    fixed + variable biases of the reference on one layout, with and without
    a fixed block; 16 seeded theta vectors each."""
    rng = np.random.default_rng(11)
    for name, fixed_blocks in (("msld_maps", ()), ("msld_maps_fixed", (6,))):
        fixed = np.zeros(13, np.uint8)
        for b in fixed_blocks:
            fixed[b] = 1
        fb = rng.normal(0, 3, 13).astype(np.float32)
        fb[0] = 0
        vb = msld_varbias(rng)
        ref = refgpu.RefMsld(MSLD_BOUND, MSLD_SITE, 5.5, fixed, fb, vb)
        th = rng.uniform(-np.pi, np.pi, (16, 13))
        th[:, 6] = np.where(fixed[6], 0.15, th[:, 6])           # a fixed block holds its lambda in theta
        lam = np.stack([ref.lambda_from_theta(t) for t in th])
        lforce = rng.normal(0, 20, (16, 13)).astype(np.float32)
        tforce = np.stack([ref.theta_force(lam[k].astype(np.float32), th[k].astype(np.float32), lforce[k])
                           for k in range(16)])
        bias = [ref.bias(lam[k].astype(np.float32)) for k in range(16)]
        np.savez_compressed(os.path.join(out, name + ".npz"), site_bound=MSLD_BOUND, lambda_site=MSLD_SITE,
                            fixed=fixed, fnex=np.float64(5.5), theta=th, lambda_ref=lam,
                            lambda_force=lforce, theta_force_ref=tforce, fixed_bias=fb,
                            var_bias=vb.view(np.uint8), bias_lambda_force_ref=np.stack([b[0] for b in bias]),
                            bias_energy_ref=np.array([b[1] for b in bias]))
        print(name, lam[0][:5], tforce[0][:5], bias[0][1], flush=True)


def update_cases(out):
    """One State::update of the reference (VVhbpR, SETTLE, OOhbpR, SETTLE,
    theta forces before and lambdas after) on the MSLD water box with rigid
    waters, friction on and the Gaussian numbers set to zero."""
    from blade_b200 import batch, holonomic
    s = systems.msld_water()
    N, nL = s.N, s.msld.blockCount
    rng = np.random.default_rng(12)
    ox = batch.water_oxygens(s)
    tri = holonomic.water_triangles(0, len(ox))
    tri["idx"] = (ox[:, None] + np.arange(3)[None, :]).astype(np.int32)
    m = batch.atom_masses(s, repartition=False)
    kT = batch.KB * 300.0
    theta_mass = batch.THETA_MASS
    vx = (rng.normal(size=(N, 3)) * np.sqrt(kT / m)[:, None]).reshape(-1)
    vt = rng.normal(size=nL) * np.sqrt(kT / theta_mass)
    th = s.msld.theta.copy()
    ref = refgpu.RefMsld(s.msld.siteBound, s.msld.lambdaSite, s.msld.fnex, n_atoms=N, box=s.box)
    lam = ref.lambda_from_theta(th)
    pos = np.concatenate([lam, s.xyz.astype(np.float64).reshape(-1), th])
    vel = np.concatenate([vx, vt]).astype(np.float32)
    fx = rng.normal(0, 5, 3 * N)
    lf = rng.normal(0, 10, nL)
    frc = np.concatenate([lf, fx, np.zeros(nL)]).astype(np.float32)
    ism = np.concatenate([np.repeat(1 / np.sqrt(m), 3), np.full(nL, 1 / np.sqrt(theta_mass))]).astype(np.float32)
    dt = 0.002 * batch.PICOSECOND
    a, at = np.exp(-1.0 / batch.PICOSECOND * dt), np.exp(-5.0 / batch.PICOSECOND * dt)
    lp = np.array([a, 0.0, 0.5 * dt, at, 0.0, 0.5 * dt], np.float32)
    p2, v2, f2 = ref.update_step(pos, vel, frc, ism, np.zeros(3 * N + nL, np.float32), lp, tri=tri, tolerance=2e-7)
    np.savez_compressed(os.path.join(out, "update_msld_water.npz"), pos_in=pos, vel_in=vel, frc_in=frc, ism=ism,
                        lp=lp, tri=tri.view(np.uint8), site_bound=s.msld.siteBound, lambda_site=s.msld.lambdaSite,
                        fnex=np.float64(s.msld.fnex), pos_ref=p2, vel_ref=v2, frc_ref=f2, n_atoms=np.int64(N))
    print("update_msld_water", N, nL, np.abs(p2 - pos).max(), flush=True)


# The reference's own CHARMM fixtures with the cutoffs their inputs use:
# test/water216/input at the 216-water configuration's 9/8 A (its default
# 10 A cutoff exceeds half the 18.856 A box), test/newDHFR/m.inp as written
# (rcut 9, rswitch 7.5, invbetaewald 3.125, orderewald 4, gridspace 1.1).
REAL = {"water216": dict(rCut=9.0, rSwitch=8.0, beta=0.34, order=6, space=1.0),
        "dhfr": dict(rCut=9.0, rSwitch=7.5, beta=0.32, order=4, space=1.1)}


def make_fixtures(reference_root, out):
    """CPU step (needs the reference's test/ tree, not a GPU): reads the PSF,
    CRD and parameter files with oracle/charmm.py and stores the systems as
    fixture_<name>.npz (blade_b200.systems.load_fixture reads them)."""
    from oracle import charmm
    for name, (psf, crd, prm, box) in charmm.fixture_paths(reference_root).items():
        c = REAL[name]
        s = charmm.build(psf, crd, prm, box, c["rCut"], c["rSwitch"], c["beta"], name)
        charmm.save_fixture(s, os.path.join(out, f"fixture_{name}.npz"))
        print("fixture", name, s.N, s.nTypes, len(s.excl), len(s.nb14), len(s.nbex), flush=True)


def real_cases(out):
    """The reference's direct space, nb14, nbex, PME reciprocal and self
    terms on the stored fixtures (GPU step)."""
    from oracle import pme_oracle
    for name, c in REAL.items():
        s = systems.load_fixture(os.path.join(HERE, f"fixture_{name}.npz"))
        ref = refgpu.RefGPU(s)
        r = ref.evaluate()
        ref.set_pairs(False)
        r14 = ref.evaluate_pairs("nb14")
        rex = ref.evaluate_pairs("nbex")
        K = [pme_oracle.grid_size(L, c["space"]) for L in s.box]
        ref.set_pme(c["order"], K)
        rp = ref.evaluate_pme("recip")
        rs = ref.evaluate_pme("self")
        f32 = lambda a: a.astype(np.float32)
        np.savez_compressed(os.path.join(out, f"real_{name}.npz"), grad=f32(r["grad"]), energy=np.float64(r["energy"]),
                            grad14=f32(r14["grad"]), energy14=np.float64(r14["energy"]),
                            gradex=f32(rex["grad"]), energyex=np.float64(rex["energy"]),
                            gradpme=f32(rp["grad"]), energypme=np.float64(rp["energy"]),
                            energyself=np.float64(rs["energy"]), K=np.int64(K), order=np.int64(c["order"]))
        print("real", name, r["energy"], r14["energy"], rex["energy"], rp["energy"], rs["energy"], K, flush=True)


def tric_cases(out):
    """The reference's triclinic direct space (State::typeBox, the flagBox
    branch of getforce_nbdirect and Domdec) on the triclinic water box, plain
    and with two MSLD sites."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_gpu_triclinic import CASES
    for name, make in CASES.items():
        s = make()
        r = refgpu.RefGPU(s).evaluate()
        np.savez_compressed(os.path.join(out, f"tric_{name}.npz"), case=np.str_(name), xyz=s.xyz.astype(np.float32),
                            grad=r["grad"].astype(np.float32), energy=np.float64(r["energy"]),
                            lambdaForce=r["lambdaForce"].astype(np.float64), tric_box=s.tric_box())
        print("tric", name, s.N, r["energy"], flush=True)


def tric_pme_cases(out):
    """The reference's triclinic PME reciprocal space (the flagBox branch of
    getforce_ewald with State::kTricBox_f) on the same two cells, order 6,
    grids from the 1 A rule on the edge lengths."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import pme_oracle
    from test_gpu_triclinic import CASES
    for name, make in CASES.items():
        s = make()
        K = [pme_oracle.grid_size(L, 1.0) for L in pme_oracle.edge_lengths(s.box6())]
        ref = refgpu.RefGPU(s)
        ref.set_pme(6, K)
        r = ref.evaluate_pme("recip")
        np.savez_compressed(os.path.join(out, f"tric_pme_{name}.npz"), case=np.str_(name),
                            xyz=s.xyz.astype(np.float32), grad=r["grad"].astype(np.float32),
                            energy=np.float64(r["energy"]), lambdaForce=r["lambdaForce"].astype(np.float64),
                            K=np.int64(K), order=np.int64(6), tric_box=s.tric_box())
        print("tric_pme", name, K, r["energy"], flush=True)


def main(out, pairs_only=False, pme_only=False, holonomic_only=False, msld_only=False, real_only=False,
         tric_only=False, tric_pme_only=False):
    os.makedirs(out, exist_ok=True)
    if tric_pme_only:
        tric_pme_cases(out)
        return
    if tric_only:
        tric_cases(out)
        tric_pme_cases(out)
        return
    if real_only:
        real_cases(out)
        return
    if holonomic_only:
        holonomic_cases(out)
        return
    if msld_only:
        msld_cases(out)
        update_cases(out)
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
    if "--fixtures" in sys.argv:
        make_fixtures(args[0], args[1] if len(args) > 1 else HERE)
        sys.exit(0)
    main(args[0] if args else os.path.join(ROOT, "golden_out"), pairs_only="--pairs-only" in sys.argv,
         pme_only="--pme-only" in sys.argv, holonomic_only="--holonomic-only" in sys.argv,
         msld_only="--msld-only" in sys.argv, real_only="--real-only" in sys.argv,
         tric_only="--tric-only" in sys.argv, tric_pme_only="--tric-pme-only" in sys.argv)
