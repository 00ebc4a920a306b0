"""Sweeps of the reference's shell script as one batch
(cuopo_batch_create_inputs): every instance with its own argv-level inputs,
2 and 3 equations, CW and nanosecond regimes, different crystals, lengths,
grating periods, modulator settings and grid sizes in one batch.

Each instance is checked against the single-instance entry point started
from the same noise: bit-identical signal and signal power (same kernel
path, same tables); FP64 instances against the FP64 CPU oracle (1e-10)."""
import numpy as np
import pytest

import cuopo_b200 as cu
from cuopo_b200 import sweep
from oracle import binding as ob
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SIGMA = 1e-3


def mixed_sweep():
    ppln = cu.default_inputs(crystal=cu.PPLN, n_eqs=2, n_z=5, lp_nm=532.0, lambda_um=6.970206862971646,
                             r_percent=95.0, mod_depth_pi=0.6, freq_det_mhz=4.0)
    spplt = cu.default_inputs(crystal=cu.SPPLT, n_eqs=3, n_z=4, lp_nm=532.0, ls_nm=1550.0,
                              lambda_um=8.719670871908674, r_percent=97.0)
    a = sweep.script_sweep(ppln, lambda_um=[6.970206862971646, 6.99], lcr_mm=[5.0, 8.0], n_thr=[2.0, 4.0],
                           delta=[0.0, 0.05], gdd_percent=[0.0, 40.0], use_eom=[0, 1], n_t=[1024, 2048])
    b = sweep.script_sweep(spplt, n_thr=[2.0, 3.0], lcr_mm=[10.0, 20.0], gdd_percent=[0.0, 30.0], n_t=[1024, 16384])
    return a + b


def signals(batch):
    out = np.zeros(batch.total, np.complex64 if batch.precision == cu.F32 else np.complex128)
    batch.get_signal(out)
    torch.cuda.synchronize()
    offs = np.concatenate([[0], np.cumsum(batch.n_t)])
    return [out[offs[k]:offs[k + 1]] for k in range(batch.count)]


def test_script_sweep_is_the_cartesian_product():
    xs = sweep.script_sweep(cu.default_inputs(), n_thr=[2.0, 3.0], lcr_mm=[5.0, 10.0, 20.0])
    assert [(x.n_thr, x.lcr_mm) for x in xs] == [(a, b) for a in (2.0, 3.0) for b in (5.0, 10.0, 20.0)]


def test_batch_of_inputs_matches_single_instance_calls():
    ins = mixed_sweep()
    seeds = np.arange(len(ins)) + 100
    n_rt = 4
    with cu.Batch(None, ins, seeds=seeds) as b:
        b.seed_noise(SIGMA)
        b.run(n_rt, 0.0)
        ps, rts, flags = b.results()
        got = signals(b)
    assert (rts == n_rt).all()
    for k, inp in enumerate(ins):
        p, _ = cu.derive_params(inp)
        with cu.Plan(p) as plan:
            Ap = torch.zeros(p.n_t, dtype=torch.complex64, device="cuda")
            As = torch.from_numpy(cu.noise_host(p.n_t, SIGMA, int(seeds[k]), 0)).cuda()
            Ai = torch.from_numpy(cu.noise_host(p.n_t, SIGMA, int(seeds[k]), 1)).cuda() if p.n_eqs == 3 else None
            hist = torch.zeros(n_rt, dtype=torch.float64, device="cuda")
            plan.round_trips(Ap, As, Ai, None, 0, 0, n_rt, ps_hist=hist)
            torch.cuda.synchronize()
            assert np.array_equal(As.cpu().numpy(), got[k]), k
            assert hist[-1].item() == ps[k], k


def test_fp64_batch_of_inputs_vs_oracle():
    ins = [cu.default_inputs(crystal=cu.PPLN, n_eqs=2, n_z=4, n_t=1024, lambda_um=6.99, lcr_mm=7.0, n_thr=3.0,
                             r_percent=93.0, delta=0.03, gdd_percent=50.0, use_eom=1, mod_depth_pi=0.6,
                             freq_det_mhz=4.0),
           cu.default_inputs(crystal=cu.SPPLT, n_eqs=3, n_z=4, n_t=1024, lp_nm=532.0, ls_nm=1550.0,
                             lambda_um=8.719670871908674, lcr_mm=15.0, n_thr=2.5, gdd_percent=20.0)]
    n_rt = 3
    rng = np.random.default_rng(5)
    starts = [(0.2 * (rng.standard_normal(1024) + 1j * rng.standard_normal(1024)),
               0.2 * (rng.standard_normal(1024) + 1j * rng.standard_normal(1024))) for _ in ins]
    with cu.Batch(None, ins, precision=cu.F64) as b:
        b.set_signal(np.concatenate([s for s, _ in starts]).astype(np.complex128))
        # the 3-equation instance starts from a zero idler (the batch's buffers start at zero)
        b.run(n_rt, 0.0)
        got = signals(b)
    for k, inp in enumerate(ins):
        p, _ = cu.derive_params(inp)
        T, w = cu.make_grids(p.n_t, p.t_rt)
        A = [np.zeros(p.n_t, np.complex128), starts[k][0].copy(),
             np.zeros(p.n_t, np.complex128) if p.n_eqs == 3 else None]
        pump = np.full(p.n_t, np.float32(p.ap0), np.complex128)
        ob.round_trips(p, w.astype(np.float64), T.astype(np.float64), A[0], A[1], A[2], pump, n_rt, 0, n_rt)
        assert rel_l2(got[k], A[1]) < 1e-10, k


def test_nanosecond_batch_matches_single_instance_calls():
    """Nanosecond 3-wave instances with different pump ratios, pulse widths,
    crystal lengths and pump windows: each runs its own window (ReadPump
    offsets included) for its n_rt round trips; fields and the power per
    round trip equal single-instance runs bit for bit."""
    base = cu.default_inputs(crystal=cu.SPPLT, n_eqs=3, regime=cu.NS, n_t=1024, n_z=4, lp_nm=532.0, ls_nm=1550.0,
                             lambda_um=8.719670871908674, r_percent=97.0)
    ins = sweep.script_sweep(base, n_thr=[2.0, 3.0], lcr_mm=[10.0, 20.0], n_rt=[5, 8])
    for k, x in enumerate(ins):
        x.fwhm_ps = 2000.0 + 500.0 * k
    seeds = np.arange(len(ins)) + 7
    with cu.Batch(None, ins, seeds=seeds) as b:
        b.seed_noise(SIGMA)
        b.run(50, 0.0)           # each instance stops at its own n_rt
        ps, rts, flags = b.results()
        got = signals(b)
        hist = [b.history(k, ins[k].n_rt) for k in range(len(ins))]
    assert [int(r) for r in rts] == [x.n_rt for x in ins]
    for k, inp in enumerate(ins):
        p, _ = cu.derive_params(inp)
        pump = cu.pump_ns(p.n_t, inp.n_rt, p.t_rt, p.ap0, inp.fwhm_ps)
        with cu.Plan(p) as plan:
            Ap = torch.zeros(p.n_t, dtype=torch.complex64, device="cuda")
            As = torch.from_numpy(cu.noise_host(p.n_t, SIGMA, int(seeds[k]), 0)).cuda()
            Ai = torch.from_numpy(cu.noise_host(p.n_t, SIGMA, int(seeds[k]), 1)).cuda()
            h = torch.zeros(inp.n_rt, dtype=torch.float64, device="cuda")
            plan.round_trips(Ap, As, Ai, torch.from_numpy(pump).cuda(), inp.n_rt, 0, inp.n_rt, ps_hist=h)
            torch.cuda.synchronize()
            assert np.array_equal(As.cpu().numpy(), got[k]), k
            assert np.array_equal(h.cpu().numpy(), hist[k]), k


def test_rejections():
    p, _ = cu.derive_params(cu.default_inputs(regime=cu.NS, n_t=1024, n_z=2))
    with pytest.raises(cu.CuopoError) as e:        # base + instances cannot carry a pump window
        cu.Batch(p, [dict(n_t=1024, ap0=p.ap0, Rs=0.98, delta=0.0, gdd=0.0, seed=0)])
    assert e.value.status == cu.EUNSUPPORTED
    with pytest.raises(cu.CuopoError) as e:
        cu.Batch(None, [cu.default_inputs(n_t=3000, n_z=2)])
    assert e.value.status == cu.EINVAL
    with cu.Batch(None, [cu.default_inputs(n_t=1024, n_z=2)]) as b, pytest.raises(cu.CuopoError):
        b.history(0, 4)                            # CW instances keep no history
