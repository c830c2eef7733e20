"""Measurements of the MSLD and batched configurations (one JSON line each).

    python -m blade_b200.suite msld   [--steps K]   # MSLD water box: pairs/s, parity, reference CUDA
    python -m blade_b200.suite batch  [--replicas R --steps K]   # batched vs one-at-a-time ns/day
    python -m blade_b200.suite alf    [...]         # learned vs plain flattening (see blade_b200.alf)

``bench.py`` carries the headline metric (the 23,558-atom system); this module
covers the other rows of the same metric.  Timings are device time from CUDA
events on the launching stream; the batched comparison reports aggregate
ns/day = replicas x steps x 2 fs / time.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

from . import systems


def _gen_replica(args):
    seed, n, sites, subs = args
    return systems.msld_chain(seed, n, sites, subs)


def batch_replicas(n_rep=64, seed=4, workers=None):
    """systems.batch_replicas, generated in parallel (spawned workers, no CUDA in them)."""
    rng = np.random.default_rng(seed)
    specs = []
    for r in range(n_rep):
        n = int(round(np.exp(rng.uniform(np.log(3000), np.log(30000)))))
        ns = int(rng.integers(1, 4))
        subs = [int(k) for k in rng.integers(2, 6, ns)]
        specs.append((seed * 1000 + r, n, ns, subs))
    workers = workers or min(16, os.cpu_count() or 1)
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_gen_replica, specs))


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_msld(args):
    import torch
    import oracle
    from oracle import refgpu
    from .nbdirect import NbDirect
    s = systems.msld_water()
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    lam = nb.lambdas_tensor()
    nb.update_domdec(pos, True)
    nb.set_counting(True)
    f64, l64, e64 = nb.evaluate(pos, lam)
    pairs = nb.pair_count()
    nb.set_counting(False)
    o = oracle.nbdirect(s)
    g = f64.cpu().numpy()
    ferr = float(np.sqrt(((g - o["grad"]) ** 2).sum() / (o["grad"] ** 2).sum()))
    lf = l64.cpu().numpy()
    lerr = float(np.sqrt(((lf[1:] - o["lambdaForce"][1:]) ** 2).sum() / (o["lambdaForce"][1:] ** 2).sum()))
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
    line = {"config": "msld_water (216-water box + 3 sites x 4 substituents, soft core)", "atoms": s.N,
            "lambda_blocks": s.msld.blockCount, "pairs_per_eval": pairs, "pairs_oracle": o["pairs"],
            "force_rel_rms_vs_fp64": ferr, "dUdlambda_rel_rms_vs_fp64": lerr,
            "bnb": {"pairs_per_s": pairs * K / t, "ms_per_step": 1e3 * t / K}}
    if refgpu.available():
        ref = refgpu.RefGPU(s)
        r = ref.evaluate()
        line["reference_vs_fp64"] = {
            "force_rel_rms": float(np.sqrt(((r["grad"] - o["grad"]) ** 2).sum() / (o["grad"] ** 2).sum())),
            "dUdlambda_rel_rms": float(np.sqrt(((r["lambdaForce"][1:] - o["lambdaForce"][1:]) ** 2).sum()
                                               / (o["lambdaForce"][1:] ** 2).sum()))}
        frames = pos.double().repeat(K, 1)
        ref.time(frames[:10], 10, 10, 10)
        t_ref = ref.time(frames, K, 10, 10) / 1e3
        line["reference_cuda"] = {"pairs_per_s": pairs * K / t_ref, "ms_per_step": 1e3 * t_ref / K}
    nb.close()
    print(json.dumps(line), flush=True)


def run_batch(args):
    import torch
    from .batch import MsldBatch, ns_per_day
    t0 = time.time()
    reps = batch_replicas(args.replicas, seed=args.seed)
    gen_s = time.time() - t0
    atoms = [r.N for r in reps]
    K = args.steps
    # batched: one handle, autotuned, one CUDA graph per 10 steps
    B = MsldBatch(reps, tune=True)
    tuning = B.tuning()
    B.capture()
    B.run_graph(20)
    torch.cuda.synchronize()
    a, b = _events()
    a.record()
    B.run_graph(K)
    b.record()
    torch.cuda.synchronize()
    t_batch = a.elapsed_time(b) / 1e3
    st, nan = B.check()
    B.close()
    del B
    torch.cuda.empty_cache()
    # one at a time: the same kernels, one replica per launch sequence
    t_seq = 0.0
    t_seq_graph = 0.0
    bad = 0
    for r in reps:
        S = MsldBatch([r], tune=args.tune_sequential)
        S.run_eager(10)
        torch.cuda.synchronize()
        a, b = _events()
        a.record()
        S.run_eager(K)
        b.record()
        torch.cuda.synchronize()
        t_seq += a.elapsed_time(b) / 1e3
        S.capture()
        torch.cuda.synchronize()
        a.record()
        S.run_graph(K)
        b.record()
        torch.cuda.synchronize()
        t_seq_graph += a.elapsed_time(b) / 1e3
        s1, n1 = S.check()
        bad += int(s1 != 0 or n1 != 0)
        S.close()
    R = len(reps)
    line = {"config": f"{R} MSLD replicas, 3k-30k atoms (log-uniform), 1-3 sites x 2-5 substituents, "
                      "rCut 12, PME+VFSWITCH, soft core, dt 2 fs",
            "replicas": R, "atoms_total": int(sum(atoms)), "atoms_min": min(atoms), "atoms_max": max(atoms),
            "steps": K, "step": "rebuild/10 + nbdirect(MSLD) + dU/dlambda->dU/dtheta + Langevin VRORV(x, theta) "
                                "+ harmonic bonds + theta->lambda; no PME recip, angles, dihedrals or SHAKE",
            "batched_graph": {"seconds": t_batch, "ns_per_day_aggregate": ns_per_day(K, t_batch, replicas=R),
                              "tuning": tuning, "status": st, "nan": nan},
            "sequential_eager": {"seconds": t_seq, "ns_per_day_aggregate": ns_per_day(K, t_seq, replicas=R)},
            "sequential_graph": {"seconds": t_seq_graph,
                                 "ns_per_day_aggregate": ns_per_day(K, t_seq_graph, replicas=R)},
            "speedup_batched_vs_sequential_eager": t_seq / t_batch,
            "speedup_batched_vs_sequential_graph": t_seq_graph / t_batch,
            "sequential_replicas_with_bad_status": bad, "generation_seconds": gen_s}
    print(json.dumps(line), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["msld", "batch", "alf"])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--tune-sequential", action="store_true")
    args, rest = ap.parse_known_args(argv)
    if args.what == "msld":
        run_msld(args)
    elif args.what == "batch":
        run_batch(args)
    else:
        from . import alf
        alf.main(rest)


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    main()
