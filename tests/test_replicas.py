"""Whole replicas per rank (blade_b200.replicas), on CPU: the partition of the
batched replicas over ranks and the gather of per-replica rows into the
global replica order over gloo, world size 2."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from blade_b200 import replicas  # noqa: E402
from blade_b200.suite import replica_specs, replica_weights  # noqa: E402


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8, 70])
def test_partition_covers_every_replica_once_and_balances(world):
    w = np.random.default_rng(world).lognormal(0.0, 1.0, 64)
    parts = replicas.partition(w, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    assert all(p == sorted(p) for p in parts)
    loads = [w[p].sum() for p in parts]
    # longest-processing-time bound: no rank exceeds the mean by more than the largest replica
    assert max(loads) <= sum(loads) / world + w.max() + 1e-12
    assert replicas.partition(w, world) == parts          # every rank computes the same split


def test_partition_of_the_batched_replicas():
    specs = replica_specs(64, 4)
    w = replica_weights(specs)
    assert all(a > 0 for a in w)
    # pairs grow with the atom count at fixed density
    n = [s[1] for s in specs]
    assert np.all(np.diff(np.asarray(w)[np.argsort(n)]) >= 0)
    for world in (2, 4, 8):
        parts = replicas.partition(w, world)
        assert replicas.imbalance(w, parts) < 1.1, world


def test_pair_estimate_matches_a_uniform_box():
    rng = np.random.default_rng(3)
    L, n, rc = 30.0, 2000, 6.0
    x = rng.uniform(0, L, (n, 3))
    d = x[:, None, :] - x[None, :, :]
    d -= L * np.round(d / L)
    r2 = (d * d).sum(-1)
    count = (np.triu(r2 < rc * rc, 1)).sum()
    est = replicas.pair_estimate(n, L ** 3, rc)
    assert abs(count - est) / est < 0.02


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    from blade_b200 import replicas as rp
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        w = np.random.default_rng(11).lognormal(0.0, 1.0, 13)
        parts = rp.partition(w, world)
        mine = parts[rank]
        # a per-replica row: (index, histogram of 5 bins filled from the index)
        rows = torch.stack([torch.tensor([float(i)] + [float(i * 10 + b) for b in range(5)], dtype=torch.float64)
                            for i in mine]) if mine else torch.zeros((0, 6), dtype=torch.float64)
        full = rp.gather_rows(rows, mine, len(w))
        out.put((rank, full.numpy(), [len(p) for p in parts]))
    finally:
        dist.destroy_process_group()


def test_gather_rows_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = np.array([[i] + [i * 10 + b for b in range(5)] for i in range(13)], np.float64)
    for rank, full, sizes in got:
        assert sum(sizes) == 13 and min(sizes) >= 1
        assert np.array_equal(full, expect), rank
