"""The multi-rank (replicas) path of bench.py on CPU with gloo, world size 2:
rank aggregation (slowest rank's time, summed pairs) and the reference arm
under torchrun (rank 0 alone runs and prints one JSON line)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        res = bench.aggregate_over_ranks(1.0 + rank, 2.0 + 3 * rank, 100.0 * (rank + 1), world, "cpu")
        res_no_e2e = bench.aggregate_over_ranks(0.5 * (rank + 1), None, 7.0, world, "cpu")
        out.put((rank, res, res_no_e2e))
    finally:
        dist.destroy_process_group()


def test_aggregate_over_two_ranks():
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
    for rank, res, res2 in got:
        assert res == (2.0, 5.0, 300.0)        # max time, max e2e time, summed pairs
        assert res2 == (1.0, None, 14.0)


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "2", "--warmup", "1", "--ref-seconds", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=540)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
