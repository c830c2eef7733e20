"""Batched MSLD stepping: batched == one-at-a-time bit for bit (no noise),
graph replay == eager stepping, and the step keeps the list valid."""
import numpy as np
import pytest
import torch

from blade_b200 import systems
from blade_b200.batch import MsldBatch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def reps():
    return [systems.msld_chain(40 + k, n, 1 + k % 2, [2 + k % 3] * (1 + k % 2))
            for k, n in enumerate((3000, 3400, 4100))]


def test_batched_equals_single_without_noise(cuda, reps):
    B = MsldBatch(reps, T=0.0)
    B.v.zero_()
    B.vt.zero_()
    B.run_eager(12)
    for r, s in enumerate(reps):
        S = MsldBatch([s], T=0.0)
        S.v.zero_()
        S.vt.zero_()
        S.run_eager(12)
        a0, a1 = 3 * B.nb.starts[r], 3 * B.nb.starts[r + 1]
        l0, l1 = B.nb.lam_starts[r], B.nb.lam_starts[r + 1]
        assert torch.equal(B.x[a0:a1], S.x)
        assert torch.equal(B.theta[l0:l1], S.theta)
        assert S.check() == (0, 0)
        S.close()
    assert B.check() == (0, 0)
    B.close()


def test_graph_replay_equals_eager(cuda, reps):
    A = MsldBatch(reps, seed=7)
    A.run_eager(30)
    G = MsldBatch(reps, seed=7)
    G.capture()            # runs 10 warm-up steps, then records 10
    G.run_graph(20)
    torch.cuda.synchronize()
    assert torch.equal(A.x, G.x)
    assert torch.equal(A.theta, G.theta)
    assert A.check() == (0, 0) and G.check() == (0, 0)
    A.close()
    G.close()


def test_lambdas_stay_on_simplex(cuda, reps):
    B = MsldBatch(reps, seed=3)
    B.capture()
    B.run_graph(50)
    lam = B.lam.cpu().numpy()
    bound = B.site_bound.cpu().numpy()
    for s in range(len(bound) - 1):
        assert lam[bound[s]:bound[s + 1]].sum() == pytest.approx(1.0, abs=1e-12)
    assert np.isfinite(B.x.cpu().numpy()).all()
    assert B.check() == (0, 0)
    B.close()


def test_autotune_keeps_results_valid(cuda, reps):
    B = MsldBatch(reps, tune=True)
    t = B.tuning()
    assert t["tiles_per_work"] in (1, 2, 4, 8, 16, 32) and t["ctas_per_sm"] in (0, 2, 3)
    assert t["tail_items"] in (0, 2)
    B.run_eager(10)
    assert B.check() == (0, 0)
    B.close()


def test_bond_gradient_matches_numpy(cuda, reps):
    s = reps[0]
    B = MsldBatch([s], T=0.0)
    x = torch.from_numpy(s.xyz.astype(np.float64).reshape(-1) + np.random.default_rng(1).normal(0, 0.05, 3 * s.N))
    B.x.copy_(x)
    B.force.zero_()
    from blade_b200 import _lib
    from blade_b200.batch import _p
    _lib.call("bnb_bond_gradient", s.N, _p(B.bond_start), _p(B.bond_partner), _p(B.bond_param), _p(B.x),
              _p(B.force), B._s(None))
    g = B.force.cpu().numpy().reshape(-1, 3)
    xx = x.numpy().reshape(-1, 3)
    b, kb, b0 = s.bonds, s.bond_param[:, 0].astype(np.float64), s.bond_param[:, 1].astype(np.float64)
    d = xx[b[:, 0]] - xx[b[:, 1]]
    r = np.linalg.norm(d, axis=1)
    f = (kb * (r - b0) / r)[:, None] * d
    ref = np.zeros_like(xx)
    np.add.at(ref, b[:, 0], f)
    np.add.at(ref, b[:, 1], -f)
    np.testing.assert_allclose(g, ref, rtol=1e-12, atol=1e-10)
    B.close()


def test_batch_with_complete_electrostatics(cuda):
    """The batched step with 1-4 pairs, exclusion corrections, PME reciprocal
    and the self term (pme=True) and rigid waters runs eagerly and from a
    captured graph, stays finite and keeps the constraints."""
    from blade_b200.batch import MsldBatch
    reps = [systems.msld_chain(51, 3000, 1, [3]), systems.msld_chain(52, 4000, 2, [2, 3])]
    B = MsldBatch(reps, constraints=True, pme=True)
    assert B.nb.pme_grid(0) != B.nb.pme_grid(1)       # two grid sizes, two FFT plans
    B.run_eager(20)
    B.capture()
    B.run_graph(20)
    torch.cuda.synchronize()
    st, nan = B.check()
    assert st == 0 and nan == 0 and int(B.cons_status.item()) == 0
    assert bool(torch.isfinite(B.x).all()) and bool(torch.isfinite(B.energy).all())
    lam = B.lam.cpu().numpy()
    assert np.all(lam >= 0) and np.all(lam <= 1 + 1e-12)
    B.close()


def test_suite_batch_over_ranks_under_torchrun(cuda):
    """The rank path of `suite batch` (whole replicas per rank, balanced by
    estimated pairs) under torchrun with one process: the partition, the
    per-rank graph run, the max-over-ranks time and the gather of per-replica
    rows all run through NCCL with world size 1."""
    import json
    import os
    import socket
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=1", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "--module", "blade_b200.suite", "batch", "--replicas", "4",
           "--steps", "20"]
    r = subprocess.run(cmd, cwd=root, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["world"] == 1 and line["replicas"] == 4 and line["replicas_per_rank"] == [4]
    assert not line["status_bad"] and line["nan"] == 0 and line["lambda_sum_per_site_ok"]
    assert line["seconds_max_over_ranks"] > 0 and line["ns_per_day_aggregate"] > 0
