"""Wall-clock time per MD step of the reference's own program on its DHFR
benchmark input, unmodified (blade_ref) and with the libbnb drop-in
(blade_bnb), both built by oracle/dropin/Makefile.  Comparison
infrastructure: the step loop, bonded terms, PME, SHAKE and the integrator
are the reference's in both; only the direct space and its list differ.

    python oracle/dropin/measure.py [--short 1000] [--long 41000] [--repeats 2]

Per-step time = (t(long) - t(short)) / (long - short) of the wall clock, the
difference removing start-up (parsing, Potential::initialize, first list
build); the program's own "Elapsed dynamics time" (run.cu:553-567, process
CPU time around the step loop) is reported beside it."""
import argparse
import json
import os
import subprocess
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(HERE), "_ref", "dropin")


def run(binary, steps, workdir):
    text = open(os.path.join(HERE, "dynamics_dhfr.inp")).read()
    text = text.replace("@FIX@", os.path.join(OUT, "fixtures")).replace("@NSTEPS@", str(steps))
    path = os.path.join(workdir, f"dyn_{steps}.inp")
    with open(path, "w") as f:
        f.write(text)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    t0 = time.perf_counter()
    r = subprocess.run([binary, path], cwd=workdir, capture_output=True, text=True, timeout=1200, env=env)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
    own = [float(l.split(":")[1]) for l in r.stdout.splitlines() if l.startswith("Elapsed dynamics time")]
    return dt, (own[-1] if own else None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--short", type=int, default=1000)
    ap.add_argument("--long", type=int, default=41000)
    ap.add_argument("--repeats", type=int, default=2)
    a = ap.parse_args()
    res = {}
    with tempfile.TemporaryDirectory() as wd:
        for name in ("blade_ref", "blade_bnb"):
            b = os.path.join(OUT, name)
            per, own = [], []
            for _ in range(a.repeats):
                (ts, os_), (tl, ol) = run(b, a.short, wd), run(b, a.long, wd)
                per.append((tl - ts) / (a.long - a.short))
                if os_ is not None and ol is not None:
                    own.append((ol - os_) / (a.long - a.short))
            res[name] = {"ms_per_step": [1e3 * p for p in per], "best_ms_per_step": 1e3 * min(per),
                         "own_elapsed_ms_per_step": [1e3 * p for p in own]}
    res["speedup_of_the_drop_in"] = res["blade_ref"]["best_ms_per_step"] / res["blade_bnb"]["best_ms_per_step"]
    res["ns_per_day"] = {k: 0.002 * 86400 / (res[k]["best_ms_per_step"] * 1e-3) / 1e3 for k in ("blade_ref", "blade_bnb")}
    res["workload"] = ("the reference's test/newDHFR with its m.inp settings: 23,558 atoms, SHAKE hbond, PME order 4, "
                       "rCut 9, rSwitch 7.5, 2 fs Langevin steps; wall clock of the whole program, difference of two "
                       "run lengths")
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
