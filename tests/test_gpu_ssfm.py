"""GPU parity of the fused SSFM kernel (through the C ABI) against the FP64 CPU
oracle (oracle/ssfm_oracle.c) and the reference's own cuFFT build (oracle/_ref).

Tolerances (relative L2 per field):
  F64 plan vs FP64 oracle ........ 1e-10 (pass and round trips)
  F32 plan vs FP64 oracle, pass .. 5e-6
  F32 plan vs FP64 oracle, rts ... 5e-5
  F32 plan vs reference (cuFFT) .. max(5e-5, 1.5 x the reference's own distance
                                   from the FP64 oracle), and no farther from the
                                   oracle than the reference itself
The reference forms its spectral phases in float (CpxExp of a float argument,
src/headers/operators.cuh:120-126); this library forms them in FP64, so where
the phases are large (pump group-velocity term of the 3-wave NS case) the two
FP32 results differ by the reference's own rounding error.
"""
import numpy as np
import pytest

import cuopo_b200 as cu
from oracle import binding as ob
from tests.helpers import params_2eq, params_3eq, random_field, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(x, prec):
    dt = torch.complex128 if prec == cu.F64 else torch.complex64
    return torch.from_numpy(np.ascontiguousarray(x)).to("cuda", dt)


def host(t):
    return t.cpu().numpy().astype(np.complex128)


def fields(p, seed):
    n = p.n_t
    Ap = random_field(n, 0.08, seed)
    As = random_field(n, 0.3, seed + 1)
    Ai = random_field(n, 0.3, seed + 2) if p.n_eqs == 3 else None
    return Ap, As, Ai


def run_pass_gpu(p, prec, Ap, As, Ai):
    T, w = cu.make_grids(p.n_t, p.t_rt)
    with cu.Plan(p, w, T, precision=prec) as plan:
        d = [dev(a, prec) if a is not None else None for a in (Ap, As, Ai)]
        plan.crystal_pass(*d)
        torch.cuda.synchronize()
        return [host(x) if x is not None else None for x in d]


def run_pass_oracle(p, Ap, As, Ai):
    T, w = cu.make_grids(p.n_t, p.t_rt)
    A = [a.copy() if a is not None else None for a in (Ap, As, Ai)]
    ob.crystal_pass(p, w.astype(np.float64), *A)
    return A


# single-CTA grids and cluster grids (2-16 CTAs with distributed shared memory;
# FP64 3-eq 2^17: fields in global memory)
CASES_F64 = [(2, 512), (2, 1024), (2, 2048), (2, 4096), (3, 512), (3, 1024), (3, 2048), (3, 4096),
             (2, 8192), (2, 16384), (2, 32768), (2, 65536), (3, 8192), (3, 16384), (3, 32768), (3, 65536),
             (3, 131072)]
CASES_F32 = [(2, 512), (2, 1024), (2, 2048), (2, 4096), (2, 8192), (3, 512), (3, 1024), (3, 2048), (3, 4096),
             (3, 8192), (2, 16384), (2, 32768), (2, 65536), (3, 16384), (3, 32768), (3, 65536), (3, 131072)]


def make_params(neq, n_t, **kw):
    return params_2eq(n_t=n_t, **kw) if neq == 2 else params_3eq(n_t=n_t, **kw)


@pytest.mark.parametrize("neq,n_t", CASES_F64)
def test_pass_f64_vs_oracle(neq, n_t):
    p = make_params(neq, n_t, n_z=6)
    Ap, As, Ai = fields(p, 10 + n_t)
    got = run_pass_gpu(p, cu.F64, Ap, As, Ai)
    ref = run_pass_oracle(p, Ap, As, Ai)
    for g, r in zip(got, ref):
        if r is not None:
            assert rel_l2(g, r) < 1e-10


@pytest.mark.parametrize("neq,n_t", CASES_F32)
def test_pass_f32_vs_oracle(neq, n_t):
    p = make_params(neq, n_t, n_z=6)
    Ap, As, Ai = fields(p, 20 + n_t)
    got = run_pass_gpu(p, cu.F32, Ap.astype(np.complex64), As.astype(np.complex64),
                       None if Ai is None else Ai.astype(np.complex64))
    ref = run_pass_oracle(p, Ap.astype(np.complex64).astype(np.complex128),
                          As.astype(np.complex64).astype(np.complex128),
                          None if Ai is None else Ai.astype(np.complex64).astype(np.complex128))
    for g, r in zip(got, ref):
        if r is not None:
            assert rel_l2(g, r) < 5e-6


@pytest.mark.parametrize("neq,n_t", [(2, 1024), (2, 8192), (2, 32768), (3, 4096), (3, 65536)])
def test_pass_phase32_vs_oracle(neq, n_t):
    """CUOPO_F32_PHASE32 plans (phase factors from FP32 sin/cos after FP64
    argument reduction) against the FP64 oracle: the same bound per pass as
    the FP32 plans with FP64-formed phases, 5e-6 relative L2."""
    p = make_params(neq, n_t, n_z=6)
    Ap, As, Ai = fields(p, 40 + n_t)
    c = (lambda a: None if a is None else a.astype(np.complex64))
    got = run_pass_gpu(p, cu.F32_PHASE32, c(Ap), c(As), c(Ai))
    ref = run_pass_oracle(p, *[None if a is None else a.astype(np.complex128) for a in (c(Ap), c(As), c(Ai))])
    for g, r in zip(got, ref):
        if r is not None:
            assert rel_l2(g, r) < 5e-6


def run_rts(p, prec, Ap, As, Ai, pump, n_rt, rt_begin, rt_count, save_first, save_count, tol=0.0):
    T, w = cu.make_grids(p.n_t, p.t_rt)
    n = p.n_t
    with cu.Plan(p, w, T, precision=prec) as plan:
        d = [dev(a, prec) if a is not None else None for a in (Ap, As, Ai)]
        dp = dev(pump, prec)
        sv = [torch.zeros(max(save_count, 1) * n, dtype=d[0].dtype, device="cuda") for _ in range(3)]
        ps = torch.zeros(max(rt_count, 1), dtype=torch.float64, device="cuda")
        done = torch.zeros(1, dtype=torch.int32, device="cuda")
        plan.round_trips(d[0], d[1], d[2], dp, n_rt, rt_begin, rt_count, sv[0], sv[1],
                         sv[2] if p.n_eqs == 3 else None, save_first, save_count, ps, tol, done)
        torch.cuda.synchronize()
        assert plan.status() == cu.OK
        out = [host(x) if x is not None else None for x in d]
        return out, [host(s) for s in sv], ps.cpu().numpy(), int(done.item())


def run_rts_oracle(p, Ap, As, Ai, pump, n_rt, rt_begin, rt_count, save_first, save_count):
    T, w = cu.make_grids(p.n_t, p.t_rt)
    n = p.n_t
    A = [a.astype(np.complex128).copy() if a is not None else None for a in (Ap, As, Ai)]
    sv = [np.zeros(max(save_count, 1) * n, np.complex128) for _ in range(3)]
    ps = np.zeros(max(rt_count, 1))
    ob.round_trips(p, w.astype(np.float64), T.astype(np.float64), A[0], A[1], A[2], pump.astype(np.complex128),
                   n_rt, rt_begin, rt_count, sv[0], sv[1], sv[2] if p.n_eqs == 3 else None, save_first,
                   save_count, ps)
    return A, sv, ps


RT_CASES = [
    # (neq, n_t, regime, kwargs)
    (2, 1024, cu.CW, dict(delta=0.07, gdd_percent=60.0)),
    (2, 2048, cu.CW, dict(delta=-0.2, use_eom=1)),
    (2, 4096, cu.CW, dict(r_percent=92.0)),
    (3, 1024, cu.NS, dict(gdd_percent=40.0, delta=0.05)),
    (3, 2048, cu.NS, dict()),
    (3, 1024, cu.CW, dict(delta=0.1)),
    (2, 16384, cu.CW, dict(delta=0.03, gdd_percent=30.0, use_eom=1)),
    (2, 32768, cu.CW, dict(r_percent=95.0)),
    (3, 65536, cu.NS, dict(gdd_percent=20.0)),
    (3, 131072, cu.NS, dict(gdd_percent=20.0, use_eom=1, mod_depth_pi=0.6, freq_det_mhz=4.0)),
]


def rt_inputs(neq, n_t, regime, kw, seed):
    p = make_params(neq, n_t, n_z=5, regime=regime, **kw)
    n_rt = 6
    Ap, As, Ai = fields(p, seed)
    if regime == cu.NS:
        pump = cu.pump_ns(n_t, n_rt, p.t_rt, p.ap0 * 3, 2.0 * p.t_rt).astype(np.complex128)
    else:
        pump = np.full(n_t, p.ap0 * 3, np.complex128)
    return p, n_rt, Ap, As, Ai, pump


@pytest.mark.parametrize("prec", [cu.F64, cu.F32])
@pytest.mark.parametrize("neq,n_t,regime,kw", RT_CASES)
def test_round_trips_vs_oracle(prec, neq, n_t, regime, kw):

    p, n_rt, Ap, As, Ai, pump = rt_inputs(neq, n_t, regime, kw, 100 + n_t)
    c = (lambda a: None if a is None else a.astype(np.complex64).astype(np.complex128))
    if prec == cu.F32:
        Ap, As, Ai, pump = c(Ap), c(As), c(Ai), c(pump)
    # all round trips of the window (the last one exercises ReadPump's offset), save rts 2..5
    got, gsv, gps, done = run_rts(p, prec, Ap, As, Ai, pump, n_rt, 0, n_rt, 2, 4)
    ref, rsv, rps = run_rts_oracle(p, Ap, As, Ai, pump, n_rt, 0, n_rt, 2, 4)
    tol = 1e-10 if prec == cu.F64 else 5e-5
    assert done == n_rt
    for g, r in zip(got, ref):
        if r is not None:
            assert rel_l2(g, r) < tol
    for f in range(neq):
        assert rel_l2(gsv[f], rsv[f]) < tol
    assert np.max(np.abs(gps - rps) / rps) < tol


def test_round_trips_rt_begin_offset():
    """Running rts 0..2 then 3..5 equals running 0..5 (state carried in the fields)."""
    p, n_rt, Ap, As, Ai, pump = rt_inputs(3, 1024, cu.NS, {}, 7)
    a, _, _, _ = run_rts(p, cu.F64, Ap, As, Ai, pump, n_rt, 0, 6, 0, 0)
    b, _, _, _ = run_rts(p, cu.F64, Ap, As, Ai, pump, n_rt, 0, 3, 0, 0)
    b, _, _, _ = run_rts(p, cu.F64, *b, pump, n_rt, 3, 3, 0, 0)
    for x, y in zip(a, b):
        assert rel_l2(x, y) < 1e-14


def test_convergence_stop_and_nonfinite_status():
    p = params_2eq(n_t=1024, n_z=4, n_thr=6, r_percent=90)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    Ap, As, _ = fields(p, 3)
    pump = np.full(p.n_t, p.ap0, np.complex128)
    with cu.Plan(p, w, T, precision=cu.F64) as plan:
        dA = [dev(Ap, cu.F64), dev(As, cu.F64)]
        ps = torch.zeros(400, dtype=torch.float64, device="cuda")
        done = torch.zeros(1, dtype=torch.int32, device="cuda")
        plan.round_trips(dA[0], dA[1], None, dev(pump, cu.F64), 0, 0, 400, ps_hist=ps, tol=0.5, rt_done=done)
        torch.cuda.synchronize()
        n = int(done.item())
        h = ps.cpu().numpy()[:n]
        assert 2 <= n < 400
        assert abs(h[-1] - h[-2]) < 0.5 * h[-1]
        assert all(abs(h[i] - h[i - 1]) >= 0.5 * h[i] for i in range(1, n - 1))
        bad = As.copy()
        bad[5] = np.nan
        plan.round_trips(dev(Ap, cu.F64), dev(bad, cu.F64), None, dev(pump, cu.F64), 0, 0, 3, rt_done=done)
        torch.cuda.synchronize()
        assert plan.status() == cu.ENONFINITE
        assert int(done.item()) == 1
        assert plan.status() == cu.OK


def test_noise_device_matches_host():
    n = 100_000
    h = cu.noise_host(n, 1e-15, 1234, 7)
    d = torch.zeros(n, dtype=torch.complex64, device="cuda")
    cu.noise_device(d, 1e-15, 1234, 7)
    torch.cuda.synchronize()
    g = d.cpu().numpy()
    assert np.array_equal(g.view(np.uint32), h.view(np.uint32))
    assert abs(np.std(g.real) / 1e-15 - 1) < 0.02


# ----------------------------------------------------- vs the reference build

# grids of one CTA (1024, 8192), of the 4- and 8-CTA cluster kernels the sweep runs (16384, 32768) and
# of the 16-CTA 3-wave kernels of the nanosecond configurations (65536, 131072)
REF_CASES = [(2, "ppln", 1024, cu.CW, dict(delta=0.05, gdd_percent=50.0, use_eom=1)),
             (2, "ppln", 8192, cu.CW, dict()),
             (2, "ppln", 16384, cu.CW, dict(delta=-0.3, gdd_percent=20.0)),
             (2, "ppln", 32768, cu.CW, dict(delta=0.4)),
             (3, "spplt", 1024, cu.NS, dict(gdd_percent=30.0)),
             (3, "spplt", 65536, cu.NS, dict(gdd_percent=20.0)),
             (3, "spplt", 131072, cu.NS, dict(delta=0.2))]


@pytest.mark.parametrize("neq,crystal,n_t,regime,kw", REF_CASES)
def test_round_trips_vs_reference_cufft(neq, crystal, n_t, regime, kw):
    if not ob.ref_available(crystal, n_t):
        pytest.skip("reference harness not built")
    p, n_rt, Ap, As, Ai, pump = rt_inputs(neq, n_t, regime, kw, 300 + n_t)
    c64 = (lambda a: None if a is None else a.astype(np.complex64))
    Ap, As, Ai, pump = c64(Ap), c64(As), c64(Ai), c64(pump)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    # one crystal pass: reference kernels + cuFFT vs this library (F32)
    pr = [x.copy() if x is not None else None for x in (Ap, As, Ai)]
    sv = [np.zeros(n_t, np.complex64) for _ in range(3)]
    rp = p.to_dict()
    q = cu.Params(**rp)
    ob.ref_round_trips(crystal, q, w, T, pr[0], pr[1], pr[2], pump, n_rt, 0, n_rt)
    got, _, _, _ = run_rts(q, cu.F32, Ap, As, Ai, pump, n_rt, 0, n_rt, 0, 0)
    orc, _, _ = run_rts_oracle(q, Ap, As, Ai, pump, n_rt, 0, n_rt, 0, 0)
    errs = []
    for name, g, r, o in zip(("pump", "signal", "idler"), got, pr, orc):
        if r is None:
            continue
        errs.append((name, rel_l2(g, r), rel_l2(r, o), rel_l2(g, o)))
    for name, e_ref, e_ref_vs_oracle, e_ours_vs_oracle in errs:
        assert e_ref < max(5e-5, 1.5 * e_ref_vs_oracle), errs
        # ours is no farther from the FP64 oracle than the reference's own FP32 build
        assert e_ours_vs_oracle < 1.2 * e_ref_vs_oracle + 2e-6, errs
