"""ctypes binding of the oracles (TEST INFRASTRUCTURE ONLY).

- liboracle64.so: the double-precision CPU restatement (oracle/ssfm_oracle.c);
- liboracle32.so: the same code in float (CPU timing baseline);
- oracle/_ref/libref_<crystal>_<size>.so: the reference's own SSFM code
  (headers included unchanged) built by oracle/build_ref.sh; runs on a GPU.

Only the tests, the smoke check and the benchmark's baseline legs use this
module.  The parameter block is the cuopo_params struct (its leading fields
are the oracle's parameter block).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_vp = C.c_void_p
_cache: dict[str, C.CDLL] = {}


def build() -> None:
    """Builds the C oracle, and oracle/_ref through its recipe (build_ref.sh
    finds the reference checkout, or CUOPO_REFERENCE_ROOT, and skips the
    harness when the sources are absent)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "CC=gcc"], check=True)
    subprocess.run([str(HERE / "build_ref.sh")], check=True)


def _load(path: Path) -> C.CDLL:
    key = str(path)
    if key not in _cache:
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (run oracle.binding.build())")
        _cache[key] = C.CDLL(key)
    return _cache[key]


def _oracle(bits: int = 64) -> C.CDLL:
    lib = _load(HERE / f"liboracle{bits}.so")
    lib.oracle_round_trips.restype = C.c_int
    lib.oracle_round_trips.argtypes = [_vp] * 6 + [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, C.c_int,
                                                   C.c_int, _vp]
    lib.oracle_crystal_pass.restype = C.c_int
    lib.oracle_crystal_pass.argtypes = [_vp] * 5
    lib.oracle_fft.restype = None
    lib.oracle_fft.argtypes = [C.c_int, _vp, _vp, C.c_int]
    lib.oracle_solve.restype = C.c_int
    lib.oracle_solve.argtypes = [_vp] * 7 + [C.c_int, C.c_int, C.c_double, _vp, _vp]
    return lib


def _arr(a, dtype):
    if a is None:
        return None
    assert a.dtype == dtype and a.flags.c_contiguous, (a.dtype, dtype)
    return a.ctypes.data


def fft(x: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised DFT with exponent sign (+1 = CUFFT_INVERSE, -1 = CUFFT_FORWARD)."""
    x = np.ascontiguousarray(x, np.complex128)
    out = np.zeros_like(x)
    _oracle(64).oracle_fft(x.size, x.ctypes.data, out.ctypes.data, sign)
    return out


def crystal_pass(params, w, Ap, As, Ai=None, bits: int = 64) -> None:
    """EvolutionInCrystal on numpy fields in place."""
    rt = np.float64 if bits == 64 else np.float32
    ct = np.complex128 if bits == 64 else np.complex64
    w = np.ascontiguousarray(w, rt)
    rc = _oracle(bits).oracle_crystal_pass(C.byref(params), w.ctypes.data, _arr(Ap, ct), _arr(As, ct),
                                           _arr(Ai, ct))
    assert rc == 0


def round_trips(params, w, T, Ap, As, Ai, pump, n_rt: int, rt_begin: int, rt_count: int,
                save_p=None, save_s=None, save_i=None, save_first: int = 0, save_count: int = 0,
                ps_hist=None, bits: int = 64) -> None:
    """Round trips of src/cuOPO.cu:474-610 on numpy fields in place."""
    rt = np.float64 if bits == 64 else np.float32
    ct = np.complex128 if bits == 64 else np.complex64
    w = np.ascontiguousarray(w, rt)
    T = np.ascontiguousarray(T, rt)
    pump = np.ascontiguousarray(pump, ct)
    rc = _oracle(bits).oracle_round_trips(
        C.byref(params), w.ctypes.data, T.ctypes.data, _arr(Ap, ct), _arr(As, ct), _arr(Ai, ct),
        pump.ctypes.data, n_rt, rt_begin, rt_count, _arr(save_p, ct), _arr(save_s, ct), _arr(save_i, ct),
        save_first, save_count, _arr(ps_hist, np.float64))
    assert rc == 0


def solve(params, w, T, Ap, As, Ai, pump, n_rt: int, max_rt: int, tol: float, bits: int = 64):
    """Runs to the convergence rule; returns (round trips, final power, converged)."""
    rt = np.float64 if bits == 64 else np.float32
    ct = np.complex128 if bits == 64 else np.complex64
    w = np.ascontiguousarray(w, rt)
    T = np.ascontiguousarray(T, rt)
    pump = np.ascontiguousarray(pump, ct)
    ps = C.c_double()
    conv = C.c_int()
    n = _oracle(bits).oracle_solve(C.byref(params), w.ctypes.data, T.ctypes.data, _arr(Ap, ct), _arr(As, ct),
                                   _arr(Ai, ct), pump.ctypes.data, n_rt, max_rt, tol, C.byref(ps),
                                   C.byref(conv))
    assert n >= 0
    return n, ps.value, bool(conv.value)


# ------------------------------------------------------- reference harness

class RefParams(C.Structure):
    """The harness's ref_params block (oracle/ref_harness.cu): the leading
    fields of the solver parameter block, filled by the reference's own
    set-up code (ref_setup_cw2) without the product library."""
    _fields_ = ([(n, C.c_int) for n in ("n_eqs", "n_t", "n_z", "regime")] +
                [(n, C.c_double) for n in ("vp", "vs", "vi", "b2p", "b2s", "b2i", "b3p", "b3s", "b3i", "dk", "kp",
                                           "ks", "ki", "dz", "alpha_crp", "alpha_crs", "alpha_cri", "Rs", "Ri",
                                           "delta", "gdd", "tod_s", "tod_i")] +
                [("use_eom", C.c_int), ("eom_idler", C.c_int), ("mod_depth", C.c_double), ("fpm", C.c_double)])


def ref_lib(crystal: str, size: int) -> C.CDLL:
    """The reference's own code (oracle/_ref) for crystal 'ppln'/'spplt' and grid size."""
    lib = _load(REF_DIR / f"libref_{crystal}_{size}.so")
    for name in ("ref_n", "ref_dndl", "ref_d2ndl2", "ref_d3ndl3", "ref_GV", "ref_GVD", "ref_TOD"):
        f = getattr(lib, name)
        f.restype = C.c_float
        f.argtypes = [C.c_float, C.c_float]
    lib.ref_dQ.restype = C.c_float
    lib.ref_deff.restype = C.c_float
    lib.ref_alpha.restype = C.c_float
    lib.ref_alpha.argtypes = [C.c_int]
    lib.ref_find_pm_temp.restype = C.c_float
    lib.ref_find_pm_temp.argtypes = [C.c_float] * 5
    lib.ref_linspace.restype = None
    lib.ref_linspace.argtypes = [_vp, C.c_int, C.c_float, C.c_float]
    lib.ref_fftshift.restype = None
    lib.ref_fftshift.argtypes = [_vp, _vp, C.c_int]
    lib.ref_input_field_cw.restype = None
    lib.ref_input_field_cw.argtypes = [_vp, C.c_float, C.c_int]
    lib.ref_input_field_gauss.restype = None
    lib.ref_input_field_gauss.argtypes = [_vp, C.c_float, _vp, C.c_float, C.c_int]
    lib.ref_size.restype = C.c_int
    lib.ref_setup_cw2.restype = None
    lib.ref_setup_cw2.argtypes = [C.c_double] * 7 + [C.c_int, _vp, _vp, _vp, _vp, _vp, _vp]
    lib.ref_round_trips.restype = C.c_int
    lib.ref_round_trips.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp,
                                    C.c_int, C.c_int, _vp, C.c_double, _vp, _vp]
    return lib


def ref_setup_cw2(size: int, lp_nm: float, lambda_um: float, n_thr: float, r_percent: float, delta_pi: float,
                  gdd_ps2: float, lcr_mm: float, n_z: int):
    """The reference's own 2-equation CW set-up (src/cuOPO.cu:92-234) for a
    MgO:PPLN grid of `size` points: returns (RefParams, w, T, pump, t_rt, ap0)."""
    lib = ref_lib("ppln", size)
    p = RefParams()
    w = np.zeros(size, np.float32)
    T = np.zeros(size, np.float32)
    pump = np.zeros(size, np.complex64)
    t_rt = C.c_double()
    ap0 = C.c_double()
    lib.ref_setup_cw2(lp_nm, lambda_um, n_thr, r_percent, delta_pi, gdd_ps2, lcr_mm, n_z, C.byref(p),
                      w.ctypes.data, T.ctypes.data, pump.ctypes.data, C.byref(t_rt), C.byref(ap0))
    return p, w, T, pump, t_rt.value, ap0.value


def ref_available(crystal: str, size: int) -> bool:
    return (REF_DIR / f"libref_{crystal}_{size}.so").exists()


def ref_round_trips(crystal: str, params, w, T, Ap, As, Ai, pump, n_rt: int, rt_begin: int, rt_count: int,
                    save_p=None, save_s=None, save_i=None, save_first: int = 0, save_count: int = 0,
                    ps_hist=None, tol: float = 0.0):
    """Runs the reference's kernels + cuFFT on the GPU (host arrays, complex64).
    Returns (rts run, loop time in ms)."""
    lib = ref_lib(crystal, params.n_t)
    w = np.ascontiguousarray(w, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    pump = np.ascontiguousarray(pump, np.complex64)
    done = C.c_int()
    ms = C.c_float()
    rc = lib.ref_round_trips(C.byref(params), w.ctypes.data, T.ctypes.data, _arr(Ap, np.complex64),
                             _arr(As, np.complex64), _arr(Ai, np.complex64), pump.ctypes.data, n_rt, rt_begin,
                             rt_count, _arr(save_p, np.complex64), _arr(save_s, np.complex64),
                             _arr(save_i, np.complex64), save_first, save_count, _arr(ps_hist, np.float64), tol,
                             C.byref(done), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference harness failed with CUDA error {rc}")
    return done.value, ms.value
