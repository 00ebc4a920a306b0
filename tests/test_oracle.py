"""CPU oracle self-checks (no GPU): the FFT against numpy, the SSFM pass against an
independent numpy restatement of src/headers/cwes2.cuh / cwes3.cuh, and analytic
properties of the cavity map."""
import numpy as np
import pytest

import cuopo_b200 as cu
from oracle import binding as ob
from tests.helpers import params_2eq, params_3eq, random_field, rel_l2


@pytest.mark.parametrize("n", [16, 256, 1024, 8192])
def test_fft_matches_numpy(n):
    x = random_field(n, 1.0, n)
    assert rel_l2(ob.fft(x, -1), np.fft.fft(x)) < 1e-13
    assert rel_l2(ob.fft(x, +1), np.fft.ifft(x) * n) < 1e-13


def np_pass(p, w, Ap, As, Ai=None):
    """Independent numpy restatement of EvolutionInCrystal (cwes2.cuh:132-215,
    cwes3.cuh:139-225), quirks Q1-Q4 included."""
    Ap, As = Ap.copy(), As.copy()
    Ai = None if Ai is None else Ai.copy()
    three = p.n_eqs == 3
    dz = p.dz
    n = p.n_t
    w = np.asarray(w, np.float64)
    if three:
        gv = [(1 / p.vp - 1 / p.vi), 0.0, (1 / p.vi - 1 / p.vs)]
    else:
        gv = [(1 / p.vp - 1 / p.vs), 0.0]
    b2 = [p.b2p, p.b2s, p.b2i]
    al = [p.alpha_crp, p.alpha_crs, p.alpha_cri]
    D = [np.exp(1j * dz * w * (gv[f] + 0.5 * w * b2[f])) * np.exp(-0.5 * al[f] * dz) for f in range(len(gv))]

    def f2(Ap, As, z):
        return (1j * p.kp * As * As * np.exp(1j * p.dk * z), 1j * p.ks * Ap * np.conj(As) * np.exp(-1j * p.dk * z))

    def f3(Ap, As, Ai, z):
        return (1j * p.kp * As * Ai * np.exp(-1j * p.dk * z), 1j * p.ks * Ap * np.conj(Ai) * np.exp(1j * p.dk * z),
                1j * p.ki * Ap * np.conj(As) * np.exp(1j * p.dk * z))

    def half(F, z):
        h = dz / 2
        if three:
            k1 = f3(*F, z); k2 = f3(*F, z + dz / 4); k3 = f3(*F, z + dz / 4); k4 = f3(*F, z + dz / 2)
        else:
            k1 = f2(*F, z)
            k2 = f2(*[a + 0.5 * k for a, k in zip(F, k1)], z + dz / 4)
            k3 = f2(*[a + 0.5 * k for a, k in zip(F, k2)], z + dz / 4)
            k4 = f2(*[a + k for a, k in zip(F, k3)], z + dz / 2)
        return [a + (q1 + 2 * q2 + 2 * q3 + q4) * h / 6 for a, q1, q2, q3, q4 in zip(F, k1, k2, k3, k4)]

    F = [Ap, As] + ([Ai] if three else [])
    z = 0.0
    for _ in range(p.n_z):
        F = half(F, z)
        F = [np.fft.fft(np.fft.ifft(a) * d) for a, d in zip(F, D)]
        F = half(F, z)
        z += dz
    return F


@pytest.mark.parametrize("three", [False, True])
def test_oracle_pass_matches_numpy_restatement(three):
    p = params_3eq(n_t=512, n_z=6) if three else params_2eq(n_t=512, n_z=6)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    Ap = random_field(p.n_t, 0.1, 1)
    As = random_field(p.n_t, 0.3, 2)
    Ai = random_field(p.n_t, 0.3, 3) if three else None
    ref = np_pass(p, w, Ap, As, Ai)
    ob.crystal_pass(p, w.astype(np.float64), Ap, As, Ai)
    got = [Ap, As] + ([Ai] if three else [])
    for g, r in zip(got, ref):
        assert rel_l2(g, r) < 1e-12


def test_pure_dispersion_is_unitary():
    """kappa = 0, alpha = 0: the pass is a product of unit-modulus spectral phases."""
    p = params_2eq(n_t=1024, n_z=10)
    p.kp = p.ks = 0.0
    p.alpha_crp = p.alpha_crs = 0.0
    T, w = cu.make_grids(p.n_t, p.t_rt)
    Ap = random_field(p.n_t, 0.1, 4)
    As = random_field(p.n_t, 0.3, 5)
    e0 = (np.sum(np.abs(Ap) ** 2), np.sum(np.abs(As) ** 2))
    ob.crystal_pass(p, w.astype(np.float64), Ap, As)
    assert abs(np.sum(np.abs(Ap) ** 2) / e0[0] - 1) < 1e-12
    assert abs(np.sum(np.abs(As) ** 2) / e0[1] - 1) < 1e-12


def test_add_phase_known_answer():
    """kappa = 0, no dispersion, no absorption: n round trips give R^{n/2} e^{i pi delta n}."""
    p = params_2eq(n_t=256, n_z=2, r_percent=95.0, delta=0.13)
    p.kp = p.ks = 0.0
    p.alpha_crp = p.alpha_crs = 0.0
    p.vp = p.vs
    p.b2p = p.b2s = 0.0
    T, w = cu.make_grids(p.n_t, p.t_rt)
    As0 = random_field(p.n_t, 0.3, 6)
    As = As0.copy()
    Ap = np.zeros(p.n_t, np.complex128)
    pump = np.full(p.n_t, 0.05, np.complex128)
    n = 7
    ob.round_trips(p, w.astype(np.float64), T.astype(np.float64), Ap, As, None, pump, 100, 0, n)
    expect = As0 * p.Rs ** (n / 2) * np.exp(1j * np.pi * p.delta * n)
    assert rel_l2(As, expect) < 1e-12
    assert np.allclose(Ap, pump)


def _manley_rowe_violation(n_z):
    p = params_3eq(n_t=256, n_z=n_z, regime=cu.CW)
    p.alpha_crp = p.alpha_crs = p.alpha_cri = 0.0
    p.b2p = p.b2s = p.b2i = 0.0
    p.vp = p.vi = p.vs
    p.dk = 0.0
    T, w = cu.make_grids(p.n_t, p.t_rt)
    Ap = np.full(p.n_t, 0.05, np.complex128)
    As = random_field(p.n_t, 0.01, 7)
    Ai = random_field(p.n_t, 0.01, 8)
    n0 = [np.sum(np.abs(a) ** 2) / k for a, k in ((Ap, p.kp), (As, p.ks), (Ai, p.ki))]
    ob.crystal_pass(p, w.astype(np.float64), Ap, As, Ai)
    n1 = [np.sum(np.abs(a) ** 2) / k for a, k in ((Ap, p.kp), (As, p.ks), (Ai, p.ki))]
    ds, di, dp = n1[1] - n0[1], n1[2] - n0[2], n1[0] - n0[0]
    assert ds > 0
    return abs(ds - di) / ds, abs(dp + ds) / ds


def test_manley_rowe_three_waves():
    """3 eqs, no loss/dispersion/mismatch: photon fluxes |A|^2/kappa obey Manley-Rowe
    (signal and idler gain what the pump loses) up to the integrator's error, which
    falls in proportion to the slice length (the half step of cwes3.cuh is first order
    because of quirk Q3)."""
    a = _manley_rowe_violation(40)
    b = _manley_rowe_violation(160)
    assert max(b) < 1e-3
    for x, y in zip(a, b):
        assert 3.0 < x / y < 5.0


def _steady_power(n_thr, n_t=256, n_z=10):
    p = params_2eq(n_t=n_t, n_z=n_z, n_thr=n_thr, r_percent=98.0)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    As = np.full(n_t, 1e-2 + 0j)
    Ap = np.zeros(n_t, np.complex128)
    pump = np.full(n_t, np.float32(p.ap0), np.complex128)
    rts, ps, conv = ob.solve(p, w.astype(np.float64), T.astype(np.float64), Ap, As, None, pump, 0, 20000, 1e-10)
    return rts, ps, conv


def test_dro_steady_state_scales_as_sqrt_pump_ratio():
    """Above threshold the degenerate DRO's steady-state signal power grows as
    sqrt(N) - 1 (plane-wave, non-resonant pump).  Pump ratios 1.5625, 2.25,
    4, 6.25 give 0.5 : 1 : 2 : 3; the solver (dispersion, finite slices, the
    reference's RK4) stays within 5 % of it (measured: 0.487, 2.023, 3.043)."""
    ref = _steady_power(2.25)
    assert ref[2]
    for n_thr, ratio in ((1.5625, 0.5), (4.0, 2.0), (6.25, 3.0)):
        rts, ps, conv = _steady_power(n_thr)
        assert conv
        assert abs(ps / ref[1] / ratio - 1.0) < 0.05, (n_thr, ps / ref[1])


def test_threshold():
    """Below threshold (N = 0.9) a seeded signal decays; above (N = 1.2) it
    grows (measured over 1000 round trips: x0.16 and x3.4 from round trip 10)."""
    for n_thr, grows in ((0.9, False), (1.2, True)):
        p = params_2eq(n_t=256, n_z=10, n_thr=n_thr, r_percent=98.0)
        T, w = cu.make_grids(p.n_t, p.t_rt)
        As = np.full(p.n_t, 1e-4 + 0j)
        Ap = np.zeros(p.n_t, np.complex128)
        pump = np.full(p.n_t, np.float32(p.ap0), np.complex128)
        ps = np.zeros(1000)
        ob.round_trips(p, w.astype(np.float64), T.astype(np.float64), Ap, As, None, pump, 1000, 0, 1000, ps_hist=ps)
        assert (ps[-1] > 2 * ps[10]) == grows and (ps[-1] < 0.5 * ps[10]) == (not grows), (n_thr, ps[10], ps[-1])
