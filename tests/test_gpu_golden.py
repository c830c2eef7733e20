"""libbnb (through the C ABI) against the reference's own outputs.

Same fixtures and tolerances as tests/test_golden.py: the B200 path must agree
with the reference's CUDA build to the reference's own FP32 rounding level.
"""
import os

import numpy as np
import pytest
import torch

from blade_b200.nbdirect import NbDirect
from test_golden import FILES, rel_rms, system_for, tolerances

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_gpu_matches_reference(cuda, path):
    z = np.load(path)
    s = system_for(os.path.basename(path)[:-4], z)
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    f, l, e = nb.evaluate(pos)
    torch.cuda.synchronize()
    n = int(z["n_forces"])
    ft, et, lt = tolerances(s)
    g = f.cpu().numpy()
    assert rel_rms(g[:n], z["grad"].astype(np.float64)) <= ft
    assert abs(float(e[0]) - float(z["energy"])) <= et * max(abs(float(z["energy"])), s.N)
    if s.msld is not None:
        assert rel_rms(l.cpu().numpy()[1:], z["lambdaForce"][1:]) <= lt
    nb.close()
