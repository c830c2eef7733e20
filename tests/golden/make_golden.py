"""Generates the golden vectors of tests/golden from the reference itself.

Runs the reference's own CUDA direct-space path (src/nbdirect + src/domdec,
unmodified, built into oracle/_ref/libbladeref.so by oracle/ref/Makefile) on
the seeded synthetic systems and stores coordinates, FP32 forces (dU/dx),
dU/dlambda and the nbdirect energy.  Needs a GPU:

    python tests/golden/make_golden.py OUTDIR

Cases: the 216-water box under all nine elecMethod x vdwMethod combinations,
the MSLD water box (soft core on and off), and the 23,558-atom chain-in-water
system (forces of the first 3,000 atoms kept).
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


def main(out):
    os.makedirs(out, exist_ok=True)
    for name, s, keep in cases():
        r = refgpu.RefGPU(s).evaluate()
        g = r["grad"].astype(np.float32)
        n = s.N if keep is None else keep
        np.savez_compressed(os.path.join(out, name + ".npz"), xyz=s.xyz.astype(np.float32),
                            grad=g[:n], energy=np.float64(r["energy"]),
                            lambdaForce=r["lambdaForce"].astype(np.float64), n_forces=np.int64(n),
                            elecMethod=np.int64(s.elecMethod), vdwMethod=np.int64(s.vdwMethod))
        print(name, s.N, r["energy"], flush=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "golden_out"))
