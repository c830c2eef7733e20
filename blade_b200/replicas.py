"""Whole replicas per rank: the multi-GPU form of the batched MSLD runs.

The replicas of a batched run (``blade_b200.batch.MsldBatch``) are independent
systems, so several GPUs share a run by taking whole replicas each, one
process per GPU, with no data-path collective: every rank steps its own
replicas on one handle.  The only exchanges are outside the step loop -- the
slowest rank's time, and per-replica statistics (the lambda histograms that
flattening pools) gathered into the global replica order.

* ``pair_estimate``: in-cutoff pairs of a replica from its atom count, box
  volume and cutoff (uniform density), the load measure the partition
  balances; the pair kernel's time is proportional to it.
* ``partition``: longest-processing-time assignment -- replicas by decreasing
  estimate, each to the rank with the least load so far (ties to the lower
  rank, then the lower replica index), so every rank computes the same split
  without communicating; each rank's replicas keep their global order.
* ``gather_rows``: per-replica rows held by their ranks -> the global
  [replicas, ...] array on every rank (one all_gather of the padded rows and
  one of their replica indices).
"""
from __future__ import annotations

import math

import numpy as np


def pair_estimate(n_atoms: int, volume: float, r_cut: float) -> float:
    """Expected pairs within r_cut of n_atoms at uniform density in volume."""
    return 0.5 * n_atoms * (n_atoms - 1) * (4.0 / 3.0) * math.pi * r_cut ** 3 / volume


def partition(weights, world: int):
    """Replica indices per rank (list of ``world`` ascending lists)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = np.asarray(weights, np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += w[i]
    return [sorted(x) for x in out]


def imbalance(weights, parts) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    w = np.asarray(weights, np.float64)
    loads = [w[p].sum() for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def gather_rows(local, ids, n_total: int, group=None):
    """Rows of this rank's replicas (``local``: tensor [len(ids), ...], rows in
    the order of ``ids``) -> tensor [n_total, ...] in global replica order on
    every rank.  Collective: every rank calls it with its own rows."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    n_local = torch.tensor([len(ids)], dtype=torch.int64, device=local.device)
    counts = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(counts, n_local, group=group)
    m = int(max(int(c.item()) for c in counts))
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:len(ids)] = local
    idx = torch.full((m,), -1, dtype=torch.int64, device=local.device)
    idx[:len(ids)] = torch.as_tensor(list(ids), dtype=torch.int64, device=local.device)
    rows = [torch.empty_like(pad) for _ in range(world)]
    idxs = [torch.empty_like(idx) for _ in range(world)]
    dist.all_gather(rows, pad, group=group)
    dist.all_gather(idxs, idx, group=group)
    out = torch.zeros((n_total,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    seen = torch.zeros(n_total, dtype=torch.bool, device=local.device)
    for r, k in zip(rows, idxs):
        ok = k >= 0
        kk = k[ok]
        if bool(seen[kk].any()):
            raise ValueError("a replica index arrived from two ranks")
        out[kk] = r[ok]
        seen[kk] = True
    if not bool(seen.all()):
        raise ValueError("some replica indices arrived from no rank")
    return out
