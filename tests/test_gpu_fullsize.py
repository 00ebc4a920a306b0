"""Full-size runs of the benchmark configurations that are not the sweep,
FP32 fields against the FP64 solver from the same seeded inputs.  (The FP64
GPU plans match the FP64 CPU oracle to 1e-10 at every kernel configuration,
tests/test_gpu_ssfm.py; the CPU oracle itself would need hours here.)

* single CW OPO: 2 equations, MgO:PPLN 5 mm, 532 -> 1064 nm, 4x threshold,
  R = 0.98, 2^13 points, 100 slices, 2000 round trips from 1e-20 noise
  (seed 0).  The signal is still in its exponential build-up at 2000
  round trips (power ~3e-24), the regime where rounding errors are
  amplified with the field.
* nanosecond OPO: 3 equations, MgO:sPPLT 20 mm, 532 -> 1550 nm, 10 ns
  Gaussian pump at 3x threshold, 2^16 points, 200 slices, 600 round trips,
  group-velocity mismatch, dispersion and absorption on, 1e-15 noise
  (seed 1); fields saved around the pump peak.
* precision study: the same OPO at 2^17 points, 400 slices, 1000 round
  trips (the FP64 run keeps its fields in global memory: 3 FP64 fields of
  2^17 points exceed a cluster's shared memory).

Tolerances (measured values on the B200 in brackets): signal power per
round trip 1e-4 [3e-5], output energy 1e-5 [8e-7].  Fields are compared
after removing the common phase (a constant phase offset between two runs
is physically irrelevant): the CW signal after 2000 round trips of build-up
2e-2 [5.3e-3], its power within 1e-4 [3.5e-5].  The nanosecond signal and
idler stay at the noise level (the 10 ns pump lasts ~25 of the 600 round
trips): 1e-2 [2.2e-3]; the pump 1e-3.  The precision study (2^17, 4e5
slices): output energy 1e-4 [2.3e-5], signal power per round trip 2e-3
[5.9e-4, the largest relative error being at the noise-level round trips
before and after the pulse], signal and idler 3e-2 [7.8e-3, 9.6e-3], pump
1e-3 [3.2e-6].  The field differences are the FP32 transforms' rounding in
the weak, noise-level modes, amplified by the build-up from noise: storing
each mode's slice factor with a compensation term (hi + lo) was measured
and changed none of them.  The precision study's third variant, FP32
phase factors after FP64 argument reduction (CUOPO_F32_PHASE32), is run
beside the FP32 one with its own bounds.
"""
import numpy as np
import pytest

import cuopo_b200 as cu

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def run(p, prec, Ap, As, Ai, pump, n_rt, save_first=0, save_count=0):
    T, w = cu.make_grids(p.n_t, p.t_rt)
    dt = torch.complex128 if prec == cu.F64 else torch.complex64
    d = [torch.from_numpy(x).to("cuda", dt) if x is not None else None for x in (Ap, As, Ai)]
    dp = torch.from_numpy(pump).to("cuda", dt)
    ps = torch.zeros(n_rt, dtype=torch.float64, device="cuda")
    sv = [torch.zeros(p.n_t * save_count, dtype=dt, device="cuda") if save_count and x is not None else None
          for x in (Ap, As, Ai)]
    with cu.Plan(p, w, T, precision=prec) as plan:
        plan.round_trips(d[0], d[1], d[2], dp, n_rt, 0, n_rt, save_p=sv[0], save_s=sv[1], save_i=sv[2],
                         save_first=save_first, save_count=save_count, ps_hist=ps)
        torch.cuda.synchronize()
    h = lambda x: x.cpu().numpy().astype(np.complex128) if x is not None else None
    return [h(x) for x in d], ps.cpu().numpy(), [h(x) for x in sv]


def aligned_rel(a, b):
    """Relative L2 of a against b after the best common phase."""
    ph = np.vdot(a, b)
    ph = ph / abs(ph) if abs(ph) > 0 else 1.0
    return float(np.linalg.norm(a * ph - b) / np.linalg.norm(b))


def f32(x):
    return x.astype(np.complex64).astype(np.complex128)


def test_single_cw_opo_2000_round_trips():
    n_t, n_rt = 8192, 2000
    inp = cu.default_inputs(n_t=n_t, n_z=100, n_rt=n_rt, lp_nm=532.0, lambda_um=6.970206862971646, n_thr=4.0,
                            r_percent=98.0, lcr_mm=5.0)
    p, _ = cu.derive_params(inp)
    As = cu.noise_host(n_t, 1e-20, 0, 1).astype(np.complex128)
    pump = cu.pump_cw(n_t, p.ap0).astype(np.complex128)
    zero = np.zeros(n_t, np.complex128)
    a = run(p, cu.F32, zero, f32(As), None, pump, n_rt)
    b = run(p, cu.F64, zero, As, None, pump, n_rt)
    e_ps = np.max(np.abs(a[1] - b[1]) / b[1])
    assert b[1][-1] > 1e3 * b[1][0], "the signal must have grown"
    assert e_ps < 1e-4, e_ps
    e_s = aligned_rel(a[0][1], b[0][1])
    assert e_s < 2e-2, e_s


# bounds: (output energy, signal power per round trip, signal power at the pulse peak, pump field,
#          signal and idler fields); measured on the B200 in the comments
NS_BOUNDS = {
    (65536, cu.F32): (1e-5, 1e-4, 1e-6, 1e-3, 1e-2),          # 8.2e-7, 1.1e-5, 2.3e-8, 2.2e-6, 2.8e-3
    (131072, cu.F32): (1e-4, 2e-3, 1e-5, 1e-3, 3e-2),         # 2.3e-5, 5.9e-4, 5.0e-7, 3.2e-6, 9.6e-3
    (131072, cu.F32_PHASE32): (1e-4, 2e-3, 1e-5, 1e-3, 5e-2),  # 1.1e-5, 3.8e-4, 2.8e-7, 9.5e-6, 1.5e-2
}


@pytest.mark.parametrize("n_t,n_z,n_rt", [(65536, 200, 600), (131072, 400, 1000)])
def test_nanosecond_three_wave_opo(n_t, n_z, n_rt):
    """The precision study at 2^17 runs both FP32 variants (FP64-formed
    phase factors, and FP32 phase factors after FP64 argument reduction)
    against the same FP64 run."""
    inp = cu.default_inputs(crystal=cu.SPPLT, n_eqs=3, regime=cu.NS, n_t=n_t, n_z=n_z, n_rt=n_rt, lp_nm=532.0,
                            ls_nm=1550.0, lambda_um=8.719670871908674, n_thr=3.0, r_percent=98.0, lcr_mm=20.0)
    p, _ = cu.derive_params(inp)
    As = cu.noise_host(n_t, 1e-15, 1, 1).astype(np.complex128)
    Ai = cu.noise_host(n_t, 1e-15, 1, 2).astype(np.complex128)
    pump = cu.pump_ns(n_t, n_rt, p.t_rt, p.ap0, inp.fwhm_ps).astype(np.complex128)
    zero = np.zeros(n_t, np.complex128)
    sf, sc = n_rt // 2 - 8, 16          # round trips around the pump peak
    b = run(p, cu.F64, zero, As, Ai, pump, n_rt, sf, sc)
    for prec in [pr for pr in (cu.F32, cu.F32_PHASE32) if (n_t, pr) in NS_BOUNDS]:
        a = run(p, prec, zero, f32(As), f32(Ai), f32(pump), n_rt, sf, sc)
        e_energy = abs(a[1].sum() - b[1].sum()) / b[1].sum()
        e_ps = np.max(np.abs(a[1] - b[1]) / b[1])
        pk = int(np.argmax(b[1]))
        e_peak = abs(a[1][pk] - b[1][pk]) / b[1][pk]
        errs = {}
        for f, name in enumerate(("pump", "signal", "idler")):
            for r in (0, sc // 2, sc - 1):
                x = a[2][f][r * n_t:(r + 1) * n_t]
                y = b[2][f][r * n_t:(r + 1) * n_t]
                errs[(name, sf + r)] = aligned_rel(x, y)
        print(f"n_t={n_t} precision={prec}: energy {e_energy:.2e}, signal power per rt {e_ps:.2e}, "
              f"at the peak {e_peak:.2e}, fields", {f"{k[0]}@{k[1]}": f"{e:.1e}" for k, e in errs.items()})
        b_energy, b_ps, b_peak, b_pump, b_field = NS_BOUNDS[(n_t, prec)]
        assert e_energy < b_energy, (prec, e_energy)
        assert e_ps < b_ps, (prec, e_ps)
        assert e_peak < b_peak, (prec, e_peak)
        bad = {k: e for k, e in errs.items() if e > (b_pump if k[0] == "pump" else b_field)}
        assert not bad, (prec, errs)
