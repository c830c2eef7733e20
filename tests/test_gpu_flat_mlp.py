"""What the trained flattening network gains over the plain update.

The committed network (tests/golden/flat_mlp.npz, trained by
``python -m blade_b200.suite alf`` with this library's BF16 kernels) is run
with those kernels on held-out histograms (tests/golden/flat_val.npz) of
replicas that later became flat.  One step of the network must land closer
to each site's flat parameters than one step of the plain update.  (In the
closed loop measured by the suite, this has not yet turned into fewer
iterations to flatness; the test pins the one-step gain.)"""
import os

import numpy as np
import pytest
import torch

from blade_b200 import alf
from blade_b200.mlp import BF16MLP
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load():
    w = np.load(os.path.join(GOLD, "flat_mlp.npz"))
    sizes = [int(v) for v in w["sizes"]]
    Ws = [mo.from_bf16_bits(w[f"W{l}_bf16"]).astype(np.float32) for l in range(len(sizes) - 1)]
    bs = [w[f"b{l}"].astype(np.float32) for l in range(len(sizes) - 1)]
    return sizes, Ws, bs, np.load(os.path.join(GOLD, "flat_val.npz"))


def test_network_step_beats_plain_update(cuda):
    sizes, Ws, bs, d = _load()
    X, Y, W, samples = d["X"].astype(np.float32), d["Y"], d["W"], int(d["samples"])
    net = BF16MLP(sizes, max_batch=len(X), seed=0)
    net.load({"sizes": np.array(sizes), **{f"W{l}": Ws[l] for l in range(len(Ws))},
              **{f"b{l}": bs[l] for l in range(len(bs))}})
    pred = net.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    # the kernels' output agrees with the FP64 oracle on the same BF16 weights
    _, outs = mo.mlp_forward(X.astype(np.float64), [w.astype(np.float64) for w in Ws],
                             [b.astype(np.float64) for b in bs])
    ref = outs[-1][1]
    assert np.abs(pred - ref).max() <= 2e-2 * np.abs(ref).max()
    dist = alf.distance_to_flat(X, Y, W, pred, samples)
    assert dist["samples"] >= 100
    assert dist["network"] < 0.85 * dist["plain_update"], dist
    assert dist["network"] < 0.85 * dist["no_change"], dist
