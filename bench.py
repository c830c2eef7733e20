#!/usr/bin/env python
"""Direct-space nonbonded throughput (pairs/s) on B200.

Workload (default): the protein-sized synthetic system -- a 2,489-atom
self-avoiding chain solute plus 7,023 TIP3P waters (23,558 atoms) in a
62.23 A periodic cube, PME real space (beta 0.32) + VFSWITCH LJ, rCut 12,
rSwitch 10, list pad 2 A rebuilt every 10 steps, FP32 coordinates moving by
seeded Gaussian steps of 0.01 A per step.  One step = one force evaluation
(pack + per-step recull + pair kernel + fixed-point reduction), plus the list
rebuild on every 10th step.  pairs/s = non-excluded pairs with r < rCut (the
oracle's count, checked against the kernel's own count) / device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bnb|reference]
                    [--workload chain_water_23558|dhfr]

--workload dhfr runs the reference's own test/newDHFR fixture instead (the
protein with its 35 CHARMM LJ types, at its input's rCut 9 / rSwitch 7.5),
which exercises the per-pair LJ table rather than the combination rule.

--impl reference times the reference algorithm's CPU restatement (FP64
oracle port, all host threads) on bounded samples of the same workload; the
reference has no CPU implementation of this path.  With N>1 (torchrun) every
rank runs its own replica (replicas only, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOPS_PER_PAIR = 60          # algorithmic FP32 flops per in-cutoff pair (FMA = 2)
REBUILD_EVERY = 10
ENERGY_EVERY = 10            # energy on the list-rebuild steps, forces every step
JITTER = 0.01                # A per step
DT_FS = 2.0
WORKLOADS = {
    "chain_water_23558": ("chain_water_23558: 2,489-atom chain + 7,023 TIP3P, 62.23 A cube, PME(beta 0.32)+"
                          "VFSWITCH, rCut 12 rSwitch 10, pad 2 A, list rebuild every 10 steps",
                          "synthetic (seeded chain-in-water, 23,558 atoms per GPU)"),
    "dhfr": ("dhfr_23558: the reference's test/newDHFR (5dfr.psf/5dfr.crd, par_all22_prot, 35 LJ types), "
             "62.23 A cube, PME(beta 0.32)+VFSWITCH, rCut 9 rSwitch 7.5 (its m.inp), pad 2 A, list rebuild "
             "every 10 steps",
             "the reference's own DHFR fixture (tests/golden/fixture_dhfr.npz) moved by seeded jitter"),
}
WORKLOAD = WORKLOADS["chain_water_23558"][0]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="bnb", choices=["bnb", "reference"])
    ap.add_argument("--workload", default="chain_water_23558", choices=sorted(WORKLOADS),
                    help="chain_water_23558 (the headline) or dhfr (the reference's own DHFR fixture)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref", action="store_true", help="skip the reference CUDA comparison leg")
    ap.add_argument("--no-pme", action="store_true", help="skip the PME reciprocal-space leg")
    ap.add_argument("--no-tune", action="store_true", help="keep the default tuning (no autotuner)")
    ap.add_argument("--tuning", default=None, help="T,C[,L]: fixed tiles per work item, CTAs per SM and work-list tail")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-seconds", type=float, default=60.0,
                    help="reference arm: CPU seconds for warm-up plus timed steps")
    return ap.parse_args()


def make_system(rank: int, workload: str = "chain_water_23558"):
    from blade_b200 import systems
    if workload == "dhfr":                       # every rank: the same protein, its own trajectory
        return systems.load_fixture(os.path.join(ROOT, "tests", "golden", "fixture_dhfr.npz"))
    s = systems.chain_in_water(seed=2 + rank)
    return s


def trajectory_np(s, k: int, seed: int):
    """Frame k of the seeded jitter trajectory (CPU), FP32."""
    rng = np.random.default_rng(seed)
    x = s.xyz.astype(np.float64)
    for _ in range(k):
        x = x + rng.normal(0, JITTER, x.shape)
    return x.astype(np.float32)


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML during a region
    (every millisecond; the timed loop also runs the counting pass and the
    e2e leg inside one sampler, so a short timed region still has samples)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, index: int):
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max = None
        self.samples, self.reasons = [], set()
        self._stop = threading.Event()

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for k, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(0.001)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


PROFILES = {"chain_water_23558": "pair_kernel_chain_water_23558.md", "dhfr": "pair_kernel_dhfr_23558.md"}


def ncu_profile_value(key, workload="chain_water_23558"):
    """A figure of the committed ncu summary of the workload's pair kernel (``key: value``), if any."""
    path = os.path.join(ROOT, "profiles", PROFILES[workload])
    try:
        for line in open(path):
            if line.strip().startswith(key + ":"):
                return float(line.split(":")[1].strip().split()[0])
    except OSError:
        pass
    return None


def ncu_traffic_per_launch(workload="chain_water_23558"):
    """DRAM bytes per pair-kernel launch from the committed ncu summary, if any."""
    return ncu_profile_value("traffic_bytes_per_launch", workload)


# ---------------------------------------------------------------------------
# reference arm: FP64 oracle port on the host cores
# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    import oracle
    s = make_system(0, args.workload)
    cores = os.cpu_count() or 1
    sampler = oracle.Sampler(s, nthreads=cores)
    x = s.xyz.astype(np.float64)
    t0 = time.perf_counter()
    full = sampler.run(x, 0, s.N)
    t_full = time.perf_counter() - t0
    # window per step so that warm-up + timed steps take about a minute
    budget = args.ref_seconds
    frac = min(1.0, budget / max(1e-9, (args.steps + args.warmup) * t_full))
    win = max(32, int(s.N * frac))
    rng = np.random.default_rng(7)
    for k in range(args.warmup):
        i0 = (k * win) % s.N
        sampler.run(x, i0, min(s.N, i0 + win))
    pairs = 0
    t0 = time.perf_counter()
    for k in range(args.steps):
        x = x + rng.normal(0, JITTER, x.shape)
        i0 = ((k + args.warmup) * win) % s.N
        pairs += sampler.run(x, i0, min(s.N, i0 + win))
    dt = time.perf_counter() - t0
    value = pairs / dt
    sample = f"pairs with lower atom index in a rotating window of {win}/{s.N} atoms per step"
    line = {"impl": "reference", "metric": "nbdirect pairs/s", "value": value, "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": WORKLOADS[args.workload][1],
            "config": {"workload": WORKLOADS[args.workload][0], "atoms": s.N, "pairs_full_eval": full},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def aggregate_over_ranks(t_total, t_e2e, pairs, world, device):
    """Whole-job numbers: the slowest rank's device times, the pairs of all
    ranks (every rank processes its own replica, so work adds up)."""
    if world <= 1:
        return t_total, t_e2e, pairs
    import torch
    import torch.distributed as dist
    t = torch.tensor([t_total, t_e2e if t_e2e is not None else 0.0], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    p = torch.tensor([pairs], dtype=torch.float64, device=device)
    dist.all_reduce(p, op=dist.ReduceOp.SUM)
    return float(t[0]), (float(t[1]) if t_e2e is not None else None), float(p[0])


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def run_bnb(args, rank, world):
    import torch
    import torch.distributed as dist
    from blade_b200 import _lib
    from blade_b200.nbdirect import NbDirect
    import ctypes as C

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    s = make_system(rank, args.workload)
    K, W = args.steps, args.warmup
    nb = NbDirect(s, device=dev)
    stream = torch.cuda.current_stream()

    # seeded trajectory, resident in HBM before timing
    gen = torch.Generator(device=dev).manual_seed(1234 + rank)
    x0 = torch.from_numpy(s.xyz.reshape(-1)).to(dev)
    frames = torch.empty((K + W, 3 * s.N), dtype=torch.float32, device=dev)
    cur = x0.double()
    for k in range(K + W):
        cur = cur + JITTER * torch.randn(cur.shape, generator=gen, device=dev, dtype=torch.float64)
        frames[k] = cur.float()
    force = torch.zeros(3 * s.N, dtype=torch.float32, device=dev)
    energy = torch.zeros(1, dtype=torch.float64, device=dev)

    def step(k, pos, all_energy=False):
        if k % REBUILD_EVERY == 0:
            nb.update_domdec(pos, True, asynchronous=(k > 0))
        calc_e = all_energy or k % ENERGY_EVERY == 0
        nb.getforce_nbdirect(pos, None, calc_e, force=force, energy=energy)

    # warm-up (first rebuild is synchronous and sizes the list), then the
    # autotuner picks tiles per work item x CTAs per SM on this system
    for k in range(W):
        step(k, frames[k])
    tuning = None
    if args.tuning:
        v = [int(x) for x in args.tuning.split(",")]
        nb.set_tuning(*v)
        for k in range(W):
            step(k, frames[k])
        tuning = dict(nb.tuning(), source="--tuning")
    elif not args.no_tune:
        tuning = nb.autotune(frames[0])
        for k in range(W):
            step(k, frames[k])
    torch.cuda.synchronize()
    st = nb.status(clear=True)
    if st:
        raise RuntimeError(f"device status {st} after warm-up")

    # pair counts per step (counting pass, untimed)
    nb.set_counting(True)
    pairs = []
    for k in range(W, W + K):
        step(k - W, frames[k], all_energy=True)
        pairs.append(nb.pair_count())
    nb.set_counting(False)
    P = float(sum(pairs))

    # this library's FP64 outputs on the first timed frame, checked against the
    # FP64 oracle in the CPU-baseline leg below (rank 0)
    first = None
    if rank == 0:
        nb.update_domdec(frames[W], True)
        f64, _, e64 = nb.evaluate(frames[W])
        first = (f64.cpu().numpy(), float(e64[0]))

    # L2 flush buffer (> 126 MB L2)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    nb.profile_read(reset=True)        # zeroes the library's launch counter
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)   # runs through the timed loop and the e2e leg below
    clocks.__enter__()
    for k in range(K):
        flush.zero_()
        evs[k][0].record(stream)
        step(k, frames[W + k])
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in evs]
    launches = nb.profile_read(reset=True)["kernel_launches"]
    st = nb.status(clear=True)
    if st:
        raise RuntimeError(f"device status {st} in timed region")
    t_total = sum(ms) / 1e3

    # per-kernel times (roofline, rebuild): the same K steps again with the
    # library's CUDA events around every pair launch and rebuild, kept out of
    # the timed loop above so that the events cost it nothing
    nb.profile(True)
    nb.profile_read(reset=True)
    for k in range(K):
        flush.zero_()
        step(k, frames[W + k])
    torch.cuda.synchronize()
    prof = nb.profile_read(reset=True)
    nb.profile(False)

    # e2e: through the C ABI with host buffers, copies inside the timed
    # regions.  Step k's region holds its pair work and, on a copy stream
    # beside it, the H2D of frame k+1 and the D2H of step k-1's forces and
    # energy (double-buffered); the region ends only when those copies are
    # done.  Region 0 also holds the H2D of frame 0, the last region the D2H
    # of the last step.  The outputs are overwritten (BNB_OUT_SET), so no
    # clearing launch precedes a step.
    e2e = None
    if not args.no_e2e:
        host_frames = frames.cpu().pin_memory()
        dpos = [torch.empty(3 * s.N, dtype=torch.float32, device=dev) for _ in range(2)]
        dforce = [torch.empty(3 * s.N, dtype=torch.float32, device=dev) for _ in range(2)]
        denergy = [torch.empty(1, dtype=torch.float64, device=dev) for _ in range(2)]
        hforce = [torch.empty(3 * s.N, dtype=torch.float32).pin_memory() for _ in range(2)]
        henergy = [torch.empty(1, dtype=torch.float64).pin_memory() for _ in range(2)]
        copy = torch.cuda.Stream(device=dev)
        e_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        copied = [torch.cuda.Event() for _ in range(K)]
        nb.update_domdec(frames[W], True)
        torch.cuda.synchronize()
        set_mode = _lib.BNB_OUT_SET

        def e2e_step(k, pos, f, e):
            if k % REBUILD_EVERY == 0:
                nb.update_domdec(pos, True, asynchronous=(k > 0))
            nb.getforce_nbdirect(pos, None, k % ENERGY_EVERY == 0, force=f, energy=e, mode=set_mode)

        for k in range(K):
            flush.zero_()
            e_evs[k][0].record(stream)
            copy.wait_stream(stream)
            with torch.cuda.stream(copy):
                if k == 0:
                    dpos[0].copy_(host_frames[W], non_blocking=True)
                    stream.wait_stream(copy)
                if k + 1 < K:
                    dpos[(k + 1) % 2].copy_(host_frames[W + k + 1], non_blocking=True)
                if k > 0:
                    hforce[(k - 1) % 2].copy_(dforce[(k - 1) % 2], non_blocking=True)
                    henergy[(k - 1) % 2].copy_(denergy[(k - 1) % 2], non_blocking=True)
                copied[k].record(copy)
            e2e_step(k, dpos[k % 2], dforce[k % 2], denergy[k % 2])
            stream.wait_event(copied[k])
            if k == K - 1:
                hforce[k % 2].copy_(dforce[k % 2], non_blocking=True)
                henergy[k % 2].copy_(denergy[k % 2], non_blocking=True)
            e_evs[k][1].record(stream)
        torch.cuda.synchronize()
        t_e2e = sum(a.elapsed_time(b) for a, b in e_evs) / 1e3
        e2e = {"t": t_e2e, "h2d": 4 * 3 * s.N, "d2h": 4 * 3 * s.N + 8}
    clocks.__exit__(None, None, None)

    # the reference's own CUDA path (src/nbdirect + src/domdec, unmodified,
    # oracle/_ref) on the same trajectory, same GPU, same L2 flushing
    ref_cuda = None
    if world == 1 and not args.no_ref:
        from oracle import refgpu
        if refgpu.available():
            try:
                ref = refgpu.RefGPU(s)
                fr64 = frames.double()
                ref.time(fr64[:W], W, REBUILD_EVERY, ENERGY_EVERY, flush)   # warm-up incl. first build
                t_ref = ref.time(fr64[W:], K, REBUILD_EVERY, ENERGY_EVERY, flush) / 1e3
                ref_cuda = {"value": P / t_ref, "unit": "pairs/s", "ms_per_step": 1e3 * t_ref / K,
                            "build": "reference src/nbdirect + src/domdec unmodified, nvcc -O3 "
                                     "-use_fast_math, sm_100a, driven by oracle/ref/ref_harness.cu",
                            "note": "same frames, rebuild and energy every 10 steps, 2 A pad, L2 flushed"}
                del fr64
            except Exception as exc:  # report, do not hide
                ref_cuda = {"unavailable": str(exc)}
        else:
            ref_cuda = {"unavailable": "oracle/_ref/libbladeref.so not built"}

    # the next row, PME reciprocal space on the same system (order 6, 1 A grid):
    # device time per evaluation, energy every 10th, next to the reference's
    # getforce_ewald on the same GPU (outside the headline's timed region)
    pme = None
    if world == 1 and not args.no_pme:
        nb.set_pme(order=6, grid_space=1.0)
        pos0 = frames[W]
        fp = torch.zeros(3 * s.N, dtype=torch.float32, device=dev)
        ep = torch.zeros(1, dtype=torch.float64, device=dev)
        reps = 200
        for k in range(10):
            nb.getforce_ewald(pos0, None, k % ENERGY_EVERY == 0, force=fp, energy=ep)
        # median of five blocks of 40 evaluations, so one stall of the host
        # that issues the launches does not stand for the kernels
        blocks = []
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for k in range(reps // 5):
                nb.getforce_ewald(pos0, None, k % ENERGY_EVERY == 0, force=fp, energy=ep)
            b.record(stream)
            torch.cuda.synchronize()
            blocks.append(a.elapsed_time(b) / (reps // 5))
        pme = {"grid": list(nb.pme_grid(0)), "order": 6, "ms_per_eval": float(np.median(blocks)),
               "ms_per_eval_blocks": blocks}
        if not args.no_ref:
            from oracle import refgpu
            if refgpu.available():
                try:
                    rp = refgpu.RefGPU(s)
                    rp.set_state(frames[W].double().cpu().numpy().reshape(-1, 3))
                    rp.set_pme(6, pme["grid"])
                    rp.time_pme(10, ENERGY_EVERY)
                    pme["reference_ms_per_eval"] = rp.time_pme(reps, ENERGY_EVERY) / reps
                except Exception as exc:  # report, do not hide
                    pme["reference"] = {"unavailable": str(exc)}

    t_total, t_e2e_max, P_all = aggregate_over_ranks(t_total, e2e["t"] if e2e else None, P, world, dev)

    if rank != 0:
        return
    value = P_all / t_total
    peak = C.c_double()
    _lib.call("bnb_fp32_peak", C.c_void_p(stream.cuda_stream), C.byref(peak))
    pair_s = prof["pair_ms"] / 1e3
    achieved = P * FLOPS_PER_PAIR / pair_s / 1e12
    peak_t = peak.value / 1e12
    traffic = ncu_traffic_per_launch(args.workload)
    line = {
        "metric": "nbdirect pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": 1e3 * t_total / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": WORKLOADS[args.workload][1],
        "config": {"workload": WORKLOADS[args.workload][0], "atoms": s.N, "lj_types": s.nTypes, "pairs_per_step": P / K, "jitter_A": JITTER,
                   "energy_every": ENERGY_EVERY,
                   "l2": "flushed (256 MB write) between timed steps", "parallelism": f"replicas x{world}",
                   "outputs": "dU/dx added to a device FP32 force array and the energy to an FP64 one "
                              "(the reference's semantics: atomic adds in the finalize); the e2e leg "
                              "overwrites its outputs (BNB_OUT_SET) and copies them to the host",
                   "tuning": tuning},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_t, "unit": "TFLOP/s",
                     "frac": achieved / peak_t, "traffic": traffic,
                     "kernel": "k_pair<PME,VFSWITCH> (per-launch mean over a second pass of the timed steps, CUDA events on its stream)",
                     "flops_per_pair": FLOPS_PER_PAIR, "peak_source": "measured FP32 FMA chains (bnb_fp32_peak)",
                     "mufu_pipe_pct_ncu": ncu_profile_value("mufu_pipe_pct", args.workload),
                     "pair_kernel_ms_mean": prof["pair_ms"] / max(1, prof["pair_launches"])},
        "rebuild_ms_mean": prof["rebuild_ms"] / max(1, prof["rebuilds"]),
        "ns_per_day_nbdirect_only": (K / t_total) * DT_FS * 86400 / 1e6,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    if ref_cuda is not None:
        line["reference_cuda_same_gpu"] = ref_cuda
    if pme is not None:
        line["pme_reciprocal"] = pme
    if e2e:
        line["e2e"] = {"value": P_all / t_e2e_max, "unit": "pairs/s", "h2d_bytes_per_step": e2e["h2d"],
                       "d2h_bytes_per_step": e2e["d2h"]}
    if world == 1 and not args.no_cpu:
        import oracle
        cores = os.cpu_count() or 1
        sam = oracle.Sampler(s, nthreads=cores)
        x = frames[W].cpu().numpy().reshape(-1, 3).astype(np.float64)
        n, tot, t0 = 0, 0, time.perf_counter()
        while time.perf_counter() - t0 < args.cpu_seconds and n < 50:
            tot += sam.run(x, 0, s.N)
            n += 1
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": tot / dt, "unit": "pairs/s", "cores": cores, "kind": "port",
                                "sample": f"{n} full FP64 evaluations of the first timed frame"}
        # the oracle as the checker of the same frame
        o = oracle.nbdirect(s, xyz=x.astype(np.float32))
        g, e = first
        line["parity_vs_fp64_oracle"] = {
            "force_rel_rms": float(np.sqrt(((g - o["grad"]) ** 2).sum() / (o["grad"] ** 2).sum())),
            "energy_rel": abs(e - o["energy"]) / max(abs(o["energy"]), s.N),
            "pairs_gpu": pairs[0], "pairs_oracle": o["pairs"]}
    print(json.dumps(line), flush=True)
    nb.close()


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_bnb(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
