"""Batched sweeps (cuopo_batch_*): a persistent launch per grid size, one
instance per CTA or cluster, resumable in round-trip chunks.

Checked against the single-instance entry point (bit-identical: same kernel
code path per instance), against chunked execution (bit-identical), and
against the FP64 CPU oracle (relative L2 <= 5e-5 on the signal after the
same round trips)."""
import numpy as np
import pytest

import cuopo_b200 as cu
from cuopo_b200 import sweep
from oracle import binding as ob
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def small_sweep(count, sizes, n_z=4, seed=3):
    base, insts, table = sweep.random_cw_sweep(count, seed, n_t_choices=sizes, n_z=n_z)
    return base, insts


def signals(batch):
    out = np.zeros(batch.total, np.complex64)
    batch.get_signal(out)
    torch.cuda.synchronize()
    offs = np.concatenate([[0], np.cumsum(batch.n_t)])
    return [out[offs[k]:offs[k + 1]] for k in range(batch.count)]


def test_batch_matches_single_instance_calls():
    base, insts = small_sweep(12, (1024, 2048, 16384))
    n_rt = 7
    with cu.Batch(base, insts) as b:
        b.seed_noise(1e-3)
        start = signals(b)
        b.run(n_rt, 0.0)
        ps, rts, flags = b.results()
        got = signals(b)
    assert (rts == n_rt).all() and (flags == 2).all()
    for k, inst in enumerate(insts):
        p = cu.Params(**base.to_dict())
        p.n_t, p.Rs, p.delta, p.gdd, p.ap0 = inst["n_t"], inst["Rs"], inst["delta"], inst["gdd"], inst["ap0"]
        with cu.Plan(p) as plan:
            Ap = torch.zeros(p.n_t, dtype=torch.complex64, device="cuda")
            As = torch.from_numpy(start[k].copy()).cuda()
            hist = torch.zeros(n_rt, dtype=torch.float64, device="cuda")
            plan.round_trips(Ap, As, None, None, 0, 0, n_rt, ps_hist=hist)
            torch.cuda.synchronize()
            assert np.array_equal(As.cpu().numpy(), got[k])
            assert hist[-1].item() == ps[k]


def test_chunked_steps_equal_one_run():
    base, insts = small_sweep(20, (1024, 4096, 32768))
    with cu.Batch(base, insts) as b1, cu.Batch(base, insts) as b2:
        b1.seed_noise(1e-2)
        b2.seed_noise(1e-2)
        b1.run(40, 1e-3, 2)
        b2.reset()
        for _ in range(5):
            b2.step(8, 40, 1e-3, 2)
        r1, r2 = b1.results(), b2.results()
        for x, y in zip(r1, r2):
            assert np.array_equal(x, y)
        for x, y in zip(signals(b1), signals(b2)):
            assert np.array_equal(x, y)
        assert b2.pending() == 0


def test_batch_vs_fp64_oracle():
    base, insts = small_sweep(6, (1024, 2048), n_z=5, seed=11)
    n_rt = 5
    with cu.Batch(base, insts) as b:
        b.seed_noise(0.05)
        start = signals(b)
        b.run(n_rt, 0.0)
        got = signals(b)
        ps, _, _ = b.results()
    for k, inst in enumerate(insts):
        p = cu.Params(**base.to_dict())
        p.n_t, p.Rs, p.delta, p.gdd, p.ap0 = inst["n_t"], inst["Rs"], inst["delta"], inst["gdd"], inst["ap0"]
        T, w = cu.make_grids(p.n_t, p.t_rt)
        As = start[k].astype(np.complex128)
        Ap = np.zeros(p.n_t, np.complex128)
        hist = np.zeros(n_rt)
        ob.round_trips(p, w.astype(np.float64), T.astype(np.float64), Ap, As, None,
                       np.full(p.n_t, p.ap0, np.complex128), 0, 0, n_rt, ps_hist=hist)
        assert rel_l2(got[k], As) < 5e-5
        assert abs(ps[k] - hist[-1]) < 5e-5 * hist[-1]


def test_convergence_flags_consistent():
    """Converged instances stopped at the first round trip whose relative power
    change fell below tol; the others ran to the limit."""
    base, insts = small_sweep(16, (1024,), n_z=4, seed=5)
    tol, max_rt = 2e-3, 300
    with cu.Batch(base, insts) as b:
        b.seed_noise(0.05)
        b.run(max_rt, tol, 1)
        ps, rts, flags = b.results()
    assert set(np.unique(flags)) <= {1, 2}
    assert (rts[flags == 2] == max_rt).all()
    assert (rts[flags == 1] < max_rt).all() and (rts[flags == 1] >= 2).all()
