"""Multi-rank host logic (cuopo_b200/shard.py) on CPU with 2 gloo ranks:
the instance split every rank computes, and the end-of-run reduction
(max of times, sum of counts) that bench.py uses for N > 1."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from cuopo_b200 import shard, sweep

torch = pytest.importorskip("torch")


def test_partition_covers_every_instance_once_and_balances():
    _, _, table = sweep.random_cw_sweep(256, 3)
    costs = shard.instance_cost(table)
    for world in (1, 2, 3, 8):
        parts = shard.partition(costs, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(256))
        loads = np.array([costs[p].sum() for p in parts])
        # LPT bound: no rank exceeds the mean by more than the largest single instance
        assert loads.max() - loads.mean() <= costs.max() + 1e-9
    assert [p.tolist() for p in shard.partition(costs, 4)] == [p.tolist() for p in shard.partition(costs, 4)]


def test_partition_edge_cases():
    assert [p.tolist() for p in shard.partition([], 2)] == [[], []]
    assert [p.tolist() for p in shard.partition([5.0], 3)] == [[0], [], []]
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)


def test_reduce_without_process_group_is_identity():
    t, n = shard.reduce_over_ranks([1.5, 2.5], [3, 4])
    assert t == [1.5, 2.5] and n == [3, 4]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        _, _, table = sweep.random_cw_sweep(64, 0)
        parts = shard.partition(shard.instance_cost(table), world)
        mine = parts[rank]
        # rank r "solves" its shard: time 10 + r ms, done = its instance count
        t, n = shard.reduce_over_ranks([10.0 + rank, 1.0], [len(mine), rank])
        out.put((rank, mine.tolist(), t, n))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_reduce():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, mine, t, n = q.get(timeout=120)
        res[r] = (mine, t, n)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0][0] + res[1][0]) == list(range(64))
    assert not set(res[0][0]) & set(res[1][0])
    for r in range(2):
        assert res[r][1] == [11.0, 1.0]          # max over ranks
        assert res[r][2] == [64, 1]              # sum over ranks
