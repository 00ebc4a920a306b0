"""Data-parallel training of the warm-start network (warmstart.train_data_parallel)
on CPU with 2 gloo ranks, with a stand-in network that has the same
interface (grad_step / grad_tensor / apply_adam) and the same Adam: with
each rank's batch its whole shard, the all-reduced mean gradient equals the
full-batch gradient, so both ranks end bit-for-bit where one process
training on all rows ends (float64)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


class LinearStandIn:
    """y = x W + b, mean squared error over all outputs, Adam (beta1 0.9,
    beta2 0.999, eps 1e-8) with a gradient scale -- the interface of
    warmstart.MLP's data-parallel calls, on CPU tensors in float64."""

    def __init__(self, n_in, n_out, seed=0):
        g = torch.Generator().manual_seed(seed)
        self.W = torch.randn(n_in, n_out, generator=g, dtype=torch.float64) * 0.3
        self.b = torch.zeros(n_out, dtype=torch.float64)
        self.grad = torch.zeros(self.W.numel() + self.b.numel(), dtype=torch.float64)
        self.m = torch.zeros_like(self.grad)
        self.v = torch.zeros_like(self.grad)
        self.t = 0

    def grad_step(self, x, t, loss=None):
        x, t = x.double(), t.double()
        d = x @ self.W + self.b - t
        g = 2.0 * d / d.numel()
        self.grad[: self.W.numel()] = (x.T @ g).reshape(-1)
        self.grad[self.W.numel():] = g.sum(0)
        if loss is not None:
            loss.fill_(float((d * d).mean()))

    def grad_tensor(self):
        return self.grad

    def apply_adam(self, lr, grad_scale=1.0):
        self.t += 1
        g = self.grad * grad_scale
        self.m.mul_(0.9).add_(0.1 * g)
        self.v.mul_(0.999).add_(0.001 * g * g)
        mh = self.m / (1 - 0.9 ** self.t)
        vh = self.v / (1 - 0.999 ** self.t)
        step = lr * mh / (vh.sqrt() + 1e-8)
        self.W -= step[: self.W.numel()].reshape(self.W.shape)
        self.b -= step[self.W.numel():]

    def params(self):
        return np.concatenate([self.W.numpy().ravel(), self.b.numpy()])


def _data():
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, (64, 4))
    y = np.sin(x @ rng.standard_normal((4, 6)))
    return x, y


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from cuopo_b200 import warmstart as ws
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        x, y = _data()
        net = LinearStandIn(4, 6)
        ws.train_data_parallel(net, x, y, steps=20, batch=0, lr=1e-2)
        out.put((rank, net.params()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process():
    from cuopo_b200 import warmstart as ws
    x, y = _data()
    ref = LinearStandIn(4, 6)
    ws.train_data_parallel(ref, x, y, steps=20, batch=0, lr=1e-2)
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, params = q.get(timeout=120)
        res[r] = params
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(res[0], res[1])
    assert np.allclose(res[0], ref.params(), rtol=1e-12, atol=1e-14)
