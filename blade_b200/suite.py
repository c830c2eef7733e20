"""Measurements of the batched and flattening configurations (one JSON line each).

    python -m blade_b200.suite batch  [--replicas R --steps K]   # batched vs one-at-a-time ns/day
    python -m blade_b200.suite alf    [--replicas R --steps K --iters T --rounds n --eval-iters E]
                                                    # learned vs plain flattening (blade_b200.alf)

``bench.py`` carries the headline metric (the 23,558-atom system); this module
covers the batched and learned rows.  Comparisons with the FP64 oracle and the
reference's CUDA build live in the test infrastructure (``python -m
oracle.measure water|msld|pme``).  Timings are device time from CUDA
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


def replica_specs(n_rep=64, seed=4):
    """(seed, atoms, sites, substituents per site) of the batched replicas:
    atom counts log-uniform in 3k-30k, 1-3 sites of 2-5 substituents."""
    rng = np.random.default_rng(seed)
    specs = []
    for r in range(n_rep):
        n = int(round(np.exp(rng.uniform(np.log(3000), np.log(30000)))))
        ns = int(rng.integers(1, 4))
        subs = [int(k) for k in rng.integers(2, 6, ns)]
        specs.append((seed * 1000 + r, n, ns, subs))
    return specs


def batch_replicas(n_rep=64, seed=4, workers=None, only=None):
    """systems.batch_replicas, generated in parallel (spawned workers, no CUDA
    in them); ``only``: the indices to generate (default all)."""
    specs = replica_specs(n_rep, seed)
    if only is not None:
        specs = [specs[i] for i in only]
    workers = workers or min(16, os.cpu_count() or 1)
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_gen_replica, specs))


def replica_weights(specs, r_cut=12.0):
    """Load of each replica for the partition over ranks: its estimated pairs."""
    from .replicas import pair_estimate
    return [pair_estimate(n, n / systems.MSLD_CHAIN_DENSITY, r_cut) for _, n, _, _ in specs]


def run_batch_ranks(args):
    """The batched run over the ranks of torchrun (one GPU each): whole
    replicas per rank, balanced by estimated pairs (blade_b200.replicas), each
    rank stepping its own on one handle under a CUDA graph; no collective in
    the step loop.  Rank 0 prints the slowest rank's device time and the
    aggregate ns/day of all replicas."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from .batch import MsldBatch, ns_per_day
    from .replicas import gather_rows, imbalance, partition
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    try:
        specs = replica_specs(args.replicas, args.seed)
        weights = replica_weights(specs)
        parts = partition(weights, world)
        mine = parts[rank]
        reps = batch_replicas(args.replicas, seed=args.seed, only=mine,
                              workers=max(1, min(16, os.cpu_count() or 1) // world)) if mine else []
        K = args.steps
        t_rank, st, nan, tuning = 0.0, 0, 0, None
        B = None
        if reps:
            B = MsldBatch(reps, tune=True, constraints=args.constraints, pme=args.pme)
            tuning = B.tuning()
            B.capture()
            B.run_graph(20)
        torch.cuda.synchronize()
        dist.barrier()
        if B is not None:
            a, b = _events()
            a.record()
            B.run_graph(K)
            b.record()
            torch.cuda.synchronize()
            t_rank = a.elapsed_time(b) / 1e3
            st, nan = B.check()
        dist.barrier()
        t = torch.tensor([t_rank, float(st != 0), float(nan)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        # per-replica statistics in global order: atoms and the final lambda sums
        rows = torch.zeros((len(mine), 2), dtype=torch.float64, device=dev)
        if B is not None:
            for k, r in enumerate(reps):
                rows[k, 0] = r.N
            lam = B.lam.double()
            starts = B.nb.lam_starts
            for k in range(len(reps)):
                rows[k, 1] = lam[starts[k]:starts[k + 1]].sum()
        allrows = gather_rows(rows, mine, len(specs))
        times = [torch.zeros(1, dtype=torch.float64, device=dev) for _ in range(world)]
        dist.all_gather(times, torch.tensor([t_rank], dtype=torch.float64, device=dev))
        if B is not None:
            B.close()
        if rank == 0:
            R = len(specs)
            line = {"config": f"{R} MSLD replicas over {world} ranks (whole replicas per rank, balanced by "
                              "estimated pairs), rCut 12, PME+VFSWITCH, soft core, dt 2 fs",
                    "replicas": R, "world": world, "steps": K, "scaling": "strong",
                    "replicas_per_rank": [len(p) for p in parts],
                    "estimated_load_imbalance": imbalance(weights, parts),
                    "seconds_max_over_ranks": float(t[0]), "seconds_per_rank": [float(x.item()) for x in times],
                    "ns_per_day_aggregate": ns_per_day(K, float(t[0]), replicas=R),
                    "atoms_total": int(allrows[:, 0].sum().item()),
                    "lambda_sum_per_site_ok": bool(torch.isfinite(allrows[:, 1]).all().item()),
                    "status_bad": bool(t[1] > 0), "nan": float(t[2]), "tuning_rank0": tuning}
            print(json.dumps(line), flush=True)
    finally:
        dist.destroy_process_group()


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_batch(args):
    if "RANK" in os.environ and "WORLD_SIZE" in os.environ:  # launched by torchrun
        return run_batch_ranks(args)
    import torch
    from .batch import MsldBatch, ns_per_day
    t0 = time.time()
    reps = batch_replicas(args.replicas, seed=args.seed)
    gen_s = time.time() - t0
    atoms = [r.N for r in reps]
    K = args.steps
    # batched: one handle, autotuned, one CUDA graph per 10 steps
    B = MsldBatch(reps, tune=True, constraints=args.constraints, pme=args.pme)
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
    # where a batched step's time goes: 20 eager steps with the pair kernel and
    # list rebuilds bracketed by CUDA events, and the in-cutoff pairs of one step
    B.nb.profile(True)
    a.record()
    B.run_eager(20)
    b.record()
    torch.cuda.synchronize()
    prof = B.nb.profile_read()
    B.nb.profile(False)
    B.nb.set_counting(True)
    B.enqueue_step(0)                     # an energy step: the pair counter runs in the energy kernels
    pairs = B.nb.pair_count()
    B.nb.set_counting(False)
    breakdown = {"eager_ms_per_step": a.elapsed_time(b) / 20, "pair_ms_per_step": prof["pair_ms"] / 20,
                 "rebuild_ms_per_rebuild": prof["rebuild_ms"] / max(1, prof["rebuilds"]),
                 "pairs_per_step": pairs, "pair_kernel_pairs_per_s": pairs / (prof["pair_ms"] / 20 / 1e3)}
    B.close()
    del B
    torch.cuda.empty_cache()
    # one at a time: the same kernels, one replica per launch sequence
    t_seq = 0.0
    t_seq_graph = 0.0
    bad = 0
    for r in reps:
        S = MsldBatch([r], tune=args.tune_sequential, constraints=args.constraints, pme=args.pme)
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
            "steps": K, "step": ("rebuild/10 + nbdirect(MSLD) + dU/dlambda->dU/dtheta + Langevin VRORV(x, theta) "
                                 + ("split around holonomic constraints (rigid TIP3P, true H masses) + chain bonds"
                                    if args.constraints else "+ harmonic bonds (HMR)")
                                 + (" + nb14 + nbex + PME reciprocal + Ewald self" if args.pme else "")
                                 + " + theta->lambda; no angles or dihedrals"
                                 + ("" if args.pme else ", no PME reciprocal")),
            "batched_graph": {"seconds": t_batch, "ns_per_day_aggregate": ns_per_day(K, t_batch, replicas=R),
                              "tuning": tuning, "status": st, "nan": nan, "breakdown": breakdown},
            "sequential_tuning": ("autotuned per replica" if args.tune_sequential
                                  else "default (--tune-sequential autotunes each replica: the fair baseline)"),
            "sequential_eager": {"seconds": t_seq, "ns_per_day_aggregate": ns_per_day(K, t_seq, replicas=R)},
            "sequential_graph": {"seconds": t_seq_graph,
                                 "ns_per_day_aggregate": ns_per_day(K, t_seq_graph, replicas=R)},
            "speedup_batched_vs_sequential_eager": t_seq / t_batch,
            "speedup_batched_vs_sequential_graph": t_seq_graph / t_batch,
            "sequential_replicas_with_bad_status": bad, "generation_seconds": gen_s}
    print(json.dumps(line), flush=True)


def _gen_flat(seed):
    from . import alf
    return alf.flattening_system(seed)


def flattening_replicas(seeds, workers=None):
    workers = workers or min(16, os.cpu_count() or 1)
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_gen_flat, list(seeds)))


def run_alf(args):
    """Learned vs plain flattening: plain runs on seeded training systems give
    (histogram, lookahead change) pairs; the BF16 MLP is trained on them with
    libbnb's kernels; both methods then run on held-out systems, batched."""
    import torch
    from . import alf
    t0 = time.time()
    R, K = args.replicas, args.steps
    if args.eval_only:
        return eval_alf(args, t0)
    Xs, Ys, Xv, Yv, rounds = [], [], [], [], []
    if args.data_in:                                    # pairs made by an earlier "--data-out" run
        for f in sorted(os.listdir(args.data_in)):
            if f.startswith("alf_pairs_") and f.endswith(".npz"):
                d = np.load(os.path.join(args.data_in, f))
                Xs.append(d["X"].astype(np.float32)); Ys.append(d["Y"].astype(np.float32))
                Xv.append(d["Xv"].astype(np.float32)); Yv.append(d["Yv"].astype(np.float32))
                rounds.append(json.loads(str(d["meta"])))
    for rnd in range(0 if args.data_in else args.rounds):
        reps = flattening_replicas(range(10000 + 1000 * rnd, 10000 + 1000 * rnd + R))
        drv = alf.AlfBatch(reps, steps=K, seed=11 + rnd)
        a, b = _events()
        a.record()
        recs = alf.run_sites(drv, args.iters)
        b.record()
        torch.cuda.synchronize()
        st = drv.status()
        drv.close()
        X, Y = alf.training_pairs(drv.sm, recs)
        rep = np.tile(np.arange(R), len(X) // R)
        val = rep >= int(0.9 * R)                       # last 10 % of the replicas: validation
        Xs.append(X[~val]); Ys.append(Y[~val]); Xv.append(X[val]); Yv.append(Y[val])
        itf = alf.site_iterations_to_flat([(r["site_dev"], r["site_frac"]) for r in recs])
        rounds.append({"seconds_gpu": a.elapsed_time(b) / 1e3, "status": st, "sites_flat": float((itf > 0).mean())})
        print(json.dumps({"round": rnd, **rounds[-1], "pairs": len(X), "t": time.time() - t0}), file=sys.stderr,
              flush=True)
        if args.data_out:
            os.makedirs(args.data_out, exist_ok=True)
            np.savez_compressed(os.path.join(args.data_out, f"alf_pairs_{rnd}.npz"), X=Xs[-1].astype(np.float16),
                                Y=Ys[-1], Xv=Xv[-1].astype(np.float16), Yv=Yv[-1], meta=json.dumps(rounds[-1]))
    if args.data_out:
        print(json.dumps({"pairs": int(sum(len(x) for x in Xs)), "rounds": rounds}), flush=True)
        return
    W = W_val = None
    if args.target == "flat":                           # point at each site's first flat parameters
        T_eff = args.iters - alf.LOOKAHEAD
        R_val = R - int(0.9 * R)
        Ys, Ws, Yv, Wv = [], [], [], []
        for k in range(len(Xs)):
            for src, dstY, dstW, n in ((Xs[k], Ys, Ws, R - R_val), (Xv[k], Yv, Wv, R_val)):
                y, w = alf.flat_targets(src.reshape(T_eff, n, -1))
                dstY.append(y.reshape(T_eff * n, -1))
                dstW.append(w.reshape(T_eff * n, -1))
        W, W_val = np.concatenate(Ws), np.concatenate(Wv)
    X, Y, X_val, Y_val = (np.concatenate(a) for a in (Xs, Ys, Xv, Yv))
    model = alf.new_model(seed=0)
    a, b = _events()
    if args.model_in:                                   # weights of an earlier training run
        model.load(dict(np.load(args.model_in)))
        first = last = None
        val = alf.train(model, X[:0], Y[:0], steps=0, X_val=X_val, Y_val=Y_val, W_val=W_val)[2]
        t_train = 0.0
    else:
        a.record()
        first, last, val = alf.train(model, X, Y, steps=args.train_steps, X_val=X_val, Y_val=Y_val, W=W,
                                     W_val=W_val,
                                     log=lambda st, l: print(f"train {st} {l:.5f}", file=sys.stderr, flush=True))
        b.record()
        torch.cuda.synchronize()
        t_train = a.elapsed_time(b) / 1e3
    if args.save:
        np.savez_compressed(args.save, **model.state())
    offline = None
    if W_val is not None:                               # one step toward the flat parameters, held-out data
        preds = []
        for k in range(0, len(X_val), model.max_batch):
            xb = torch.from_numpy(np.ascontiguousarray(X_val[k:k + model.max_batch])).to(model.dev)
            preds.append(model.forward(xb).cpu().numpy())
        offline = alf.distance_to_flat(X_val, Y_val, W_val, np.concatenate(preds), K)
    out = evaluate_modes(args, model, R, K)
    line = {"config": f"learned flattening: {R} batched replicas of the 216-water box + 3 sites x 4 substituents "
                      f"(variants of one fragment), {K} steps (x 2 fs) per iteration",
            "flat_criterion": f"per site: max |end-state population - 1/4| <= {alf.FLAT_TOL}, "
                              f">= {alf.END_FRAC_MIN} of samples at end states",
            "training": {"pairs": int(len(X)), "validation_pairs": int(len(X_val)), "rounds": rounds,
                         "iterations_per_round": args.iters, "lookahead": alf.LOOKAHEAD,
                         "mlp": [alf.FEAT_PAD, *alf.HIDDEN, alf.OUT_PAD], "steps": args.train_steps,
                         "loss_first": first, "loss_last": last, "loss_validation": val, "seconds_gpu": t_train},
            "step_distance_to_flat_parameters": offline,
            "eval_iterations": args.eval_iters, **out,
            "seconds_total": time.time() - t0}
    print(json.dumps(line), flush=True)


def evaluate_modes(args, model, R, K):
    """Plain and learned flattening on held-out systems (same systems, same MD
    seed): iterations until each site is first judged flat, per iteration
    and, with --pool W, on the last W iterations pooled (alf.site_flatness_pooled)."""
    from . import alf
    reps = flattening_replicas(range(50000, 50000 + R))
    out = {}
    modes = [m for m in args.eval_modes.split(",") if m]
    for name in modes:  # plain | learned:<scale> | plain+learned:<scale> | learned_first:<iterations>
        mdl = None if name == "plain" else model
        arg = float(name.split(":")[1]) if ":" in name else 1.0
        first = int(arg) if name.startswith("learned_first") else None
        drv = alf.AlfBatch(reps, steps=K, seed=99)
        recs = alf.run_sites(drv, args.eval_iters, mdl, scale=1.0 if first is not None else arg,
                             with_plain=name.startswith("plain+"), learned_iters=first, pool=args.pool)
        st = drv.status()
        drv.close()
        itf = alf.site_iterations_to_flat([(r["site_dev"], r["site_frac"]) for r in recs])
        capped = np.where(itf > 0, itf, args.eval_iters + 1)
        fb = [float(r["fallback"].mean()) for r in recs if r["fallback"] is not None]
        out[name] = {"median_iterations_to_flat": float(np.median(capped)), "mean_iterations_to_flat": float(capped.mean()),
                     "sites_flat": float((itf > 0).mean()),
                     "site_dev_median_per_iteration": [round(float(np.median(r["site_dev"])), 3) for r in recs],
                     "fallback_fraction": float(np.mean(fb)) if fb else None, "status": st}
        if args.pool > 1:
            itp = alf.site_iterations_to_flat([(r["site_dev_pool"], r["site_frac_pool"]) for r in recs])
            cp = np.where(itp > 0, itp, args.eval_iters + 1)
            out[name]["pooled"] = {"window": args.pool, "median_iterations_to_flat": float(np.median(cp)),
                                   "mean_iterations_to_flat": float(cp.mean()), "sites_flat": float((itp > 0).mean()),
                                   "site_dev_median_per_iteration":
                                       [round(float(np.median(r["site_dev_pool"])), 3) for r in recs]}
    return out


def eval_alf(args, t0):
    """Evaluation only: the network of --model-in against the plain update."""
    from . import alf
    if not args.model_in:
        raise SystemExit("--eval-only needs --model-in")
    model = alf.new_model(seed=0)
    model.load(dict(np.load(args.model_in)))
    out = evaluate_modes(args, model, args.replicas, args.steps)
    line = {"config": f"learned flattening, evaluation of {os.path.basename(args.model_in)}: {args.replicas} "
                      f"batched replicas of the 216-water box + 3 sites x 4 substituents (variants of one "
                      f"fragment), {args.steps} steps (x 2 fs) per iteration",
            "flat_criterion": f"per site: max |end-state population - 1/4| <= {alf.FLAT_TOL}, "
                              f">= {alf.END_FRAC_MIN} of samples at end states; per iteration, and pooled over "
                              f"the last {args.pool} iterations reweighted to the current biases",
            "eval_iterations": args.eval_iters, **out, "seconds_total": time.time() - t0}
    print(json.dumps(line), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["batch", "alf"])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--tune-sequential", action="store_true")
    ap.add_argument("--pool", type=int, default=0, help="alf: also judge flatness on the last POOL iterations pooled")
    ap.add_argument("--eval-only", action="store_true", help="alf: evaluate the network of --model-in only")
    ap.add_argument("--iters", type=int, default=60)
    ap.add_argument("--rounds", type=int, default=3)
    ap.add_argument("--eval-iters", type=int, default=30)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--save", default=None)
    ap.add_argument("--data-out", default=None)
    ap.add_argument("--data-in", default=None)
    ap.add_argument("--model-in", default=None)
    ap.add_argument("--eval-modes", default="plain,learned:1")
    ap.add_argument("--target", default="flat", choices=["flat", "lookahead"])
    ap.add_argument("--constraints", action="store_true", help="batch: rigid waters (holonomic constraints)")
    ap.add_argument("--pme", action="store_true", help="batch: 1-4, exclusion corrections, PME reciprocal, self")
    args, rest = ap.parse_known_args(argv)
    if args.what == "batch":
        run_batch(args)
    else:
        run_alf(args)


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    main()
