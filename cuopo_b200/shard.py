"""Multi-GPU plumbing for sweeps: one process per GPU, instances sharded, no
collective on the data path.

Sweep instances are independent (the reference runs each as its own process,
src/cuOPO.sh:91-174), so ranks never exchange fields.  Two things cross
ranks, both through torch.distributed (NCCL on GPUs, gloo on CPU): the
split of one instance list over the ranks, and the end-of-run reduction
of timings (max over ranks) and counts (sum).
"""
from __future__ import annotations

import numpy as np


def instance_cost(table, n_z: int = 100, rts=None) -> np.ndarray:
    """Relative cost of each instance: n_t log2(n_t) * n_z * expected round
    trips (the growth estimate of the sweep unless `rts` is given)."""
    from .sweep import growth_estimate
    nt = np.asarray(table["n_t"], dtype=np.float64)
    r = np.asarray(rts, dtype=np.float64) if rts is not None else np.minimum(growth_estimate(table), 5000.0)
    return nt * np.log2(nt) * n_z * r


def partition(costs, world: int) -> list[np.ndarray]:
    """Longest-processing-time split of instances over `world` ranks: each
    instance, most expensive first, goes to the rank with the least work so
    far (ties to the lower rank).  Returns each rank's instance indices in
    ascending order; deterministic, so every rank computes the same split."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    load = np.zeros(world)
    owner = np.empty(len(costs), dtype=np.int64)
    for i in np.argsort(-costs, kind="stable"):
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return [np.flatnonzero(owner == r) for r in range(world)]


def reduce_over_ranks(times_ms, counts, device=None):
    """Max over ranks of each time, sum over ranks of each count (one
    all-reduce each); identity without an initialised process group."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(times_ms), dtype=torch.float64, device=device)
    n = torch.tensor(list(counts), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.cpu()], [int(round(float(x))) for x in n.cpu()]
