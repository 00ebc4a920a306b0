"""Host set-up parity: the product's Sellmeier models, temperature scan, grids and
pump windows against the reference's own host functions (src/headers/ppln.cuh,
spplt.cuh, functions.cuh, compiled unchanged into oracle/_ref).  Bit-exact."""

import numpy as np
import pytest

import cuopo_b200 as cu
from oracle import binding as ob

pytestmark = pytest.mark.skipif(not (ob.ref_available("ppln", 1024) and ob.ref_available("spplt", 1024)),
                                reason="reference harness (oracle/_ref) not built")

CRYSTALS = [(cu.PPLN, "ppln"), (cu.SPPLT, "spplt")]
FUNCS = [(0, "ref_n"), (1, "ref_dndl"), (2, "ref_d2ndl2"), (3, "ref_d3ndl3"), (4, "ref_GV"), (5, "ref_GVD"),
         (6, "ref_TOD")]


def f32(x):
    return float(np.float32(x))


@pytest.mark.parametrize("crystal,name", CRYSTALS)
@pytest.mark.parametrize("which,fname", FUNCS)
def test_sellmeier_bit_exact(crystal, name, which, fname):
    ref = getattr(ob.ref_lib(name, 1024), fname)
    bad = []
    for L in np.linspace(0.45, 2.6, 87):
        for T in np.linspace(10.0, 150.0, 23):
            a = cu.sellmeier(crystal, which, f32(L), f32(T))
            b = ref(f32(L), f32(T))
            if not (a == b or (np.isnan(a) and np.isnan(b))):
                bad.append((L, T, a, b))
    assert not bad, bad[:5]


@pytest.mark.parametrize("crystal,name", CRYSTALS)
@pytest.mark.parametrize("lp,ls,lam", [(0.532, 1.064, 6.970206862971646), (0.532, 1.064, 7.1),
                                       (0.532, 1.55, 8.719670871908674), (1.55, 3.1, 35.01), (0.532, 1.064, 7.97)])
def test_phase_matching_temperature_scan(crystal, name, lp, ls, lam):
    ref = ob.ref_lib(name, 1024)
    a = cu.phase_matching_temp(crystal, f32(lp), f32(ls), f32(lam), 10.0, 150.0)
    b = ref.ref_find_pm_temp(f32(lp), f32(ls), f32(lam), 10.0, 150.0)
    assert a == b


@pytest.mark.parametrize("n,lo,hi", [(1024, -176.36, 176.36), (5000, 10.0, 150.0), (65536 * 3, -6e4, 6e4)])
def test_linspace_bit_exact(n, lo, hi):
    ref = ob.ref_lib("ppln", 1024)
    a = cu.linspace(n, f32(lo), f32(hi))
    b = np.zeros(n, np.float32)
    ref.ref_linspace(b.ctypes.data, n, f32(lo), f32(hi))
    assert np.array_equal(a, b)


@pytest.mark.parametrize("n_t", [512, 1024, 8192])
def test_grids_bit_exact(n_t):
    """cuOPO.cu:169-189: T = linspace, w = 2 pi fftshift(linspace(-N dF/2, N dF/2))."""
    ref = ob.ref_lib("ppln", 1024)
    t_rt = f32(352.72381591796875)
    T, w = cu.make_grids(n_t, t_rt)
    Tr = np.zeros(n_t, np.float32)
    ref.ref_linspace(Tr.ctypes.data, n_t, f32(-0.5 * t_rt), f32(0.5 * t_rt))
    dF = np.float32(1) / np.float32(t_rt)
    F = np.zeros(n_t, np.float32)
    ref.ref_linspace(F.ctypes.data, n_t, f32(-0.5 * n_t * float(dF)), f32(0.5 * n_t * float(dF)))
    wr = np.zeros(n_t, np.float32)
    ref.ref_fftshift(wr.ctypes.data, F.ctypes.data, n_t)
    wr = (np.float32(2) * np.float32(3.14159265358979323846)) * wr
    assert np.array_equal(T, Tr)
    assert np.array_equal(w, wr.astype(np.float32))


def test_ns_pump_window_bit_exact():
    """NS Gaussian window (cuOPO.cu:243-247, functions.cuh:77-85) on the float Tp grid."""
    ref = ob.ref_lib("spplt", 1024)
    n_t, n_rt, t_rt, ap0 = 1024, 40, f32(408.0742492675781), f32(0.0564594566822052)
    a = cu.pump_ns(n_t, n_rt, t_rt, ap0, 10000.0)
    T_width = np.float32(t_rt) * np.float32(n_rt)
    Tp = np.zeros(n_t * n_rt, np.float32)
    ref.ref_linspace(Tp.ctypes.data, n_t * n_rt, f32(-0.5 * float(T_width)), f32(0.5 * float(T_width)))
    sig = np.float32(10000) * np.sqrt(np.float32(2)) / (np.float32(2) * np.sqrt(np.float32(2) * np.log(np.float32(2))))
    b = np.zeros(n_t * n_rt, np.complex64)
    ref.ref_input_field_gauss(b.ctypes.data, ap0, Tp.ctypes.data, f32(sig), n_t * n_rt)
    assert np.array_equal(a, b)


def test_cw_pump():
    ref = ob.ref_lib("ppln", 1024)
    a = cu.pump_cw(1024, 0.0952628)
    b = np.zeros(1024, np.complex64)
    ref.ref_input_field_cw(b.ctypes.data, f32(0.0952628), 1024)
    assert np.array_equal(a, b)


def test_material_constants():
    for crystal, name in CRYSTALS:
        ref = ob.ref_lib(name, 1024)
        p, _ = cu.derive_params(cu.default_inputs(crystal=crystal, n_t=1024, n_z=10))
        assert p.alpha_crp == ref.ref_alpha(0) and p.alpha_crs == ref.ref_alpha(1) and p.alpha_cri == ref.ref_alpha(2)


def test_derived_c1_values():
    """C1 physics: PPLN 532 -> 1064 nm, 5 mm, Lambda for dk = 0 at 26.85 C; the scan picks T = 26.859 C."""
    p, info = cu.derive_params(cu.default_inputs(n_t=8192, n_z=100, lambda_um=6.970206862971646, n_thr=4,
                                                 r_percent=98, lcr_mm=5))
    ref = ob.ref_lib("ppln", 1024)
    T = f32(info.temp_c)
    assert p.vp == ref.ref_GV(f32(0.532), T) and p.vs == ref.ref_GV(f32(1.064), T)
    assert p.b2s == ref.ref_GVD(f32(1.064), T)
    assert abs(info.temp_c - 26.859371) < 1e-5
    assert p.dz == 50.0 and p.n_t == 8192
    assert 0.09 < p.ap0 < 0.1


@pytest.mark.parametrize("n_t", [4096, 8192, 16384, 32768])
@pytest.mark.parametrize("n_thr,r_percent,delta,gdd_fs2", [(4.0, 98.0, 0.0, 0.0), (1.37, 90.4, -0.61, 321.5),
                                                          (5.83, 98.9, 0.97, -488.0)])
def test_reference_cw_setup_matches_product(n_t, n_thr, r_percent, delta, gdd_fs2):
    """The harness's restatement of the reference's 2-equation CW set-up
    (src/cuOPO.cu:92-234, used by the benchmark's reference arm without the
    product library) equals the product's cuopo_derive_params, grids and CW
    pump bit for bit."""
    if not ob.ref_available("ppln", n_t):
        pytest.skip("reference harness not built for this grid")
    from cuopo_b200 import sweep
    p, _ = cu.derive_params(sweep.cw_base_inputs(n_t=n_t, n_z=100, n_thr=n_thr, r_percent=r_percent))
    T, w = cu.make_grids(n_t, p.t_rt)
    pump = cu.pump_cw(n_t, p.ap0)
    rp, rw, rT, rpump, t_rt, ap0 = ob.ref_setup_cw2(n_t, 532.0, 6.970206862971646, n_thr, r_percent, delta,
                                                    gdd_fs2 * 1e-6, 5.0, 100)
    for name in ("vp", "vs", "b2p", "b2s", "dk", "kp", "ks", "dz", "alpha_crp", "alpha_crs", "Rs", "Ri"):
        assert getattr(rp, name) == getattr(p, name), name
    assert rp.delta == f32(delta) and rp.gdd == f32(gdd_fs2 * 1e-6)
    assert (t_rt, ap0) == (p.t_rt, p.ap0)
    assert np.array_equal(rw, w) and np.array_equal(rT, T) and np.array_equal(rpump, pump)
