"""Measurements against the FP64 oracle and the reference's own CUDA build
(test and measurement infrastructure; the product never imports this module).

    python -m oracle.measure water [--steps K]   # 216-water box: pairs/s, parity, reference CUDA
    python -m oracle.measure msld  [--steps K]   # MSLD water box: pairs/s, parity, reference CUDA
    python -m oracle.measure pme   [--steps K] [--parts single,batch]
                                                 # PME reciprocal: time per evaluation, parity,
                                                 # reference getforce_ewald, batched replicas

Timings are device time from CUDA events on the launching stream; one JSON
line per run.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from blade_b200 import systems  # noqa: E402


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_msld(args, water_only=False):
    """One system, many evaluations: pairs/s, error against the FP64 oracle,
    and the reference's CUDA build on the same GPU.  water_only: the 216-water
    box without MSLD sites, else the MSLD box."""
    import torch
    import oracle
    from oracle import refgpu
    from blade_b200.nbdirect import NbDirect
    s = systems.water_box() if water_only else systems.msld_water()
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    lam = nb.lambdas_tensor()
    nb.update_domdec(pos, True)
    tuning = nb.autotune(pos, lam)
    nb.set_counting(True)
    f64, l64, e64 = nb.evaluate(pos, lam)
    pairs = nb.pair_count()
    nb.set_counting(False)
    o = oracle.nbdirect(s)
    g = f64.cpu().numpy()
    ferr = float(np.sqrt(((g - o["grad"]) ** 2).sum() / (o["grad"] ** 2).sum()))
    lf = l64.cpu().numpy()
    lerr = (float(np.sqrt(((lf[1:] - o["lambdaForce"][1:]) ** 2).sum() / (o["lambdaForce"][1:] ** 2).sum()))
            if s.msld else None)
    e_rel = float(abs(float(e64.cpu()[0]) - o["energy"]) / abs(o["energy"]))
    K = args.steps
    force = torch.zeros(3 * s.N, device="cuda")
    lforce = torch.zeros(nb.L, device="cuda")
    for k in range(10):
        nb.getforce_nbdirect(pos, lam, True, force=force, lambda_force=lforce)
    a, b = _events()
    a.record()
    for k in range(K):
        if k % 10 == 0:
            nb.update_domdec(pos, True, asynchronous=True)
        nb.getforce_nbdirect(pos, lam, k % 10 == 0, force=force, lambda_force=lforce)
    b.record()
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3
    line = {"config": ("water_box (216 TIP3P, 18.856 A, rc 9 / rs 8, beta 0.34)" if water_only else
                       "msld_water (216-water box + 3 sites x 4 substituents, soft core)"), "atoms": s.N,
            "lambda_blocks": s.msld.blockCount if s.msld else 1, "pairs_per_eval": pairs, "pairs_oracle": o["pairs"],
            "force_rel_rms_vs_fp64": ferr, "dUdlambda_rel_rms_vs_fp64": lerr, "energy_rel_err_vs_fp64": e_rel,
            "bnb": {"pairs_per_s": pairs * K / t, "ms_per_step": 1e3 * t / K, "tuning": tuning}}
    if refgpu.available():
        ref = refgpu.RefGPU(s)
        r = ref.evaluate()
        line["reference_vs_fp64"] = {
            "force_rel_rms": float(np.sqrt(((r["grad"] - o["grad"]) ** 2).sum() / (o["grad"] ** 2).sum())),
            "dUdlambda_rel_rms": (float(np.sqrt(((r["lambdaForce"][1:] - o["lambdaForce"][1:]) ** 2).sum()
                                                / (o["lambdaForce"][1:] ** 2).sum())) if s.msld else None)}
        frames = pos.double().repeat(K, 1)
        ref.time(frames[:10], 10, 10, 10)
        t_ref = ref.time(frames, K, 10, 10) / 1e3
        line["reference_cuda"] = {"pairs_per_s": pairs * K / t_ref, "ms_per_step": 1e3 * t_ref / K}
    nb.close()
    print(json.dumps(line), flush=True)


def run_pme(args):
    """PME reciprocal space: device time per evaluation of bnb_compute_pme and
    of the reference's getforce_ewald (its CUDA build, same GPU) on the
    23,558-atom chain-in-water system (64^3 grid, order 6) and the water box
    (20^3), error against the FP64 oracle, and the 64 batch replicas on one
    handle against one handle per replica."""
    import torch
    from oracle import pme_oracle, refgpu
    from blade_b200.nbdirect import NbDirect
    K_E = 332.0716
    out = {"config": "PME reciprocal space, order 6, grids from 1 A spacing; energy every 10th evaluation"}
    reps = args.steps

    def time_calls(fn, n):
        for k in range(10):
            fn(k)
        a, b = _events()
        a.record()
        for k in range(n):
            fn(k)
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    parts = set(args.parts.split(","))
    singles_sys = (("chain_water_23558", systems.chain_in_water()), ("water216", systems.water_box()))
    for name, s in (singles_sys if "single" in parts else ()):
        nb = NbDirect(s)
        nb.set_pme(order=6, grid_space=1.0)
        K = nb.pme_grid(0)
        pos = nb.positions_tensor()
        f64, _, e64 = nb.evaluate_pme(pos)
        E, g, _, _ = pme_oracle.pme_recip(s.xyz, s.nbonds["q"], s.box, K, 6, s.betaEwald, K_E)
        force = torch.zeros(3 * s.N, device="cuda")
        energy = torch.zeros(1, dtype=torch.float64, device="cuda")
        ms = time_calls(lambda k: nb.getforce_ewald(pos, None, k % 10 == 0, force=force, energy=energy), reps)
        line = {"atoms": s.N, "grid": K, "bnb_ms_per_eval": ms,
                "force_rel_rms_vs_fp64": float(np.sqrt(((f64.cpu().numpy() - g) ** 2).sum() / (g ** 2).sum())),
                "energy_rel_err_vs_fp64": abs(float(e64.cpu()[0]) - E) / abs(E)}
        if refgpu.available():
            ref = refgpu.RefGPU(s)
            ref.set_pme(6, K)
            r = ref.evaluate_pme("recip")
            ref.time_pme(10)
            line["reference_ms_per_eval"] = ref.time_pme(reps) / reps
            line["reference_force_rel_rms_vs_fp64"] = float(np.sqrt(((r["grad"] - g) ** 2).sum() / (g ** 2).sum()))
        out[name] = line
        nb.close()
    if "batch" not in parts:
        print(json.dumps(out), flush=True)
        return
    # batch: 64 replicas of 3k-30k atoms, one handle vs one handle per replica
    reps_sys = systems.batch_replicas(args.replicas, seed=args.seed)
    nb = NbDirect(reps_sys)
    nb.set_pme(order=6, grid_space=1.0)
    pos = nb.positions_tensor()
    lam = nb.lambdas_tensor()
    force = torch.zeros(3 * nb.N, device="cuda")
    lforce = torch.zeros(nb.L, device="cuda")
    ms_b = time_calls(lambda k: nb.getforce_ewald(pos, lam, False, force=force, lambda_force=lforce), 50)
    singles = []
    for s in reps_sys:
        one = NbDirect(s)
        one.set_pme(order=6, grid_space=1.0)
        singles.append((one, one.positions_tensor(), one.lambdas_tensor(),
                        torch.zeros(3 * s.N, device="cuda"), torch.zeros(one.L, device="cuda")))

    def all_singles(k):
        for one, p, l, f, lf in singles:
            one.getforce_ewald(p, l, False, force=f, lambda_force=lf)
    ms_s = time_calls(all_singles, 20)
    out["batch"] = {"replicas": len(reps_sys), "atoms": nb.N, "batched_ms_per_eval": ms_b,
                    "one_handle_per_replica_ms_per_eval": ms_s, "speedup": ms_s / ms_b,
                    "distinct_grids": len({tuple(nb.pme_grid(r)) for r in range(nb.R)})}
    for one, *_ in singles:
        one.close()
    nb.close()
    print(json.dumps(out), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["water", "msld", "pme"])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--parts", default="single,batch", help="pme: single (one system) and/or batch")
    args = ap.parse_args(argv)
    if args.what == "pme":
        run_pme(args)
    else:
        run_msld(args, water_only=args.what == "water")


if __name__ == "__main__":
    main()
