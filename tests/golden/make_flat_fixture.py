"""Writes the learned-flattening fixtures used by tests/test_gpu_flat_mlp.py and
tests/test_alf.py from a trained model and held-out pairs made by
``python -m blade_b200.suite alf --data-out DIR`` / ``--save MODEL``:

    python tests/golden/make_flat_fixture.py MODEL.npz DIR/alf_pairs_1.npz 128 60

flat_mlp.npz: the network's weights as BF16 bit patterns (what its kernels
use) and FP32 biases.  flat_val.npz: up to 300 held-out samples (features in
FP16, targets toward each site's first flat parameters, element weights).
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
from blade_b200 import alf  # noqa: E402
from oracle.mlp_oracle import bf16_bits  # noqa: E402

model, pairs, R, iters = sys.argv[1], sys.argv[2], int(sys.argv[3]), int(sys.argv[4])
here = os.path.dirname(os.path.abspath(__file__))
w = np.load(model)
out = {"sizes": w["sizes"]}
for l in range(len(w["sizes"]) - 1):
    out[f"W{l}_bf16"] = bf16_bits(w[f"W{l}"])
    out[f"b{l}"] = w[f"b{l}"].astype(np.float32)
np.savez_compressed(os.path.join(here, "flat_mlp.npz"), **out)
d = np.load(pairs)
T, Rv = iters - alf.LOOKAHEAD, R - int(0.9 * R)
Xv = d["Xv"].astype(np.float32)
Y, W = alf.flat_targets(Xv.reshape(T, Rv, -1))
Y, W = Y.reshape(T * Rv, -1), W.reshape(T * Rv, -1)
keep = np.nonzero(W[:, :alf.N_PARAMS_REP].any(1))[0][:300]
np.savez_compressed(os.path.join(here, "flat_val.npz"), X=Xv[keep].astype(np.float16), Y=Y[keep], W=W[keep],
                    samples=np.int64(10000))
print("wrote", len(keep), "samples")
