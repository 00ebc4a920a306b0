"""ctypes binding of libcuopo_b200.so (the C ABI declared in include/cuopo.h).

The shared library is built in-tree by cuopo_b200/build.py.  Loading fails
loudly when it is missing: there is no Python or CPU fallback for the solver.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libcuopo_b200.so"

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, ENONFINITE, EUNSUPPORTED, EIO = range(8)
PPLN, SPPLT = 0, 1
CW, NS = 0, 1
F32, F64, F32_PHASE32 = 0, 1, 2

_STATUS_NAMES = {0: "CUOPO_OK", 1: "CUOPO_EINVAL", 2: "CUOPO_ENOMEM", 3: "CUOPO_ECUDA", 4: "CUOPO_ETIMEOUT",
                 5: "CUOPO_ENONFINITE", 6: "CUOPO_EUNSUPPORTED", 7: "CUOPO_EIO"}


class CuopoError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Params(C.Structure):
    """cuopo_params (include/cuopo.h)."""
    _fields_ = [
        ("n_eqs", C.c_int), ("n_t", C.c_int), ("n_z", C.c_int), ("regime", C.c_int),
        ("vp", C.c_double), ("vs", C.c_double), ("vi", C.c_double),
        ("b2p", C.c_double), ("b2s", C.c_double), ("b2i", C.c_double),
        ("b3p", C.c_double), ("b3s", C.c_double), ("b3i", C.c_double),
        ("dk", C.c_double), ("kp", C.c_double), ("ks", C.c_double), ("ki", C.c_double), ("dz", C.c_double),
        ("alpha_crp", C.c_double), ("alpha_crs", C.c_double), ("alpha_cri", C.c_double),
        ("Rs", C.c_double), ("Ri", C.c_double), ("delta", C.c_double),
        ("gdd", C.c_double), ("tod_s", C.c_double), ("tod_i", C.c_double),
        ("use_eom", C.c_int), ("eom_idler", C.c_int),
        ("mod_depth", C.c_double), ("fpm", C.c_double),
        ("t_rt", C.c_double), ("ap0", C.c_double),
    ]

    def to_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Inputs(C.Structure):
    """cuopo_inputs (include/cuopo.h)."""
    _fields_ = [
        ("crystal", C.c_int), ("n_eqs", C.c_int), ("regime", C.c_int),
        ("n_t", C.c_int), ("n_z", C.c_int), ("n_rt", C.c_int),
        ("lp_nm", C.c_double), ("temp_c", C.c_double), ("lambda_um", C.c_double),
        ("n_thr", C.c_double), ("r_percent", C.c_double), ("delta", C.c_double),
        ("gdd_percent", C.c_double), ("tod_percent", C.c_double),
        ("use_eom", C.c_int), ("mod_depth_pi", C.c_double), ("freq_det_mhz", C.c_double),
        ("lcr_mm", C.c_double), ("ls_nm", C.c_double), ("temp_from_scan", C.c_int),
        ("lcav_um", C.c_double), ("ri", C.c_double), ("waist_um", C.c_double), ("fwhm_ps", C.c_double),
    ]


class Info(C.Structure):
    """cuopo_info (include/cuopo.h)."""
    _fields_ = [(k, C.c_double) for k in (
        "temp_c", "np", "ns", "ni", "li", "dkp", "t_rt", "fsr", "finesse", "ith", "pth", "power",
        "gamma_l", "alphas", "alphai", "sigmap", "dT", "dF")]


class Instance(C.Structure):
    """cuopo_instance (include/cuopo.h)."""
    _fields_ = [("n_t", C.c_int), ("ap0", C.c_double), ("Rs", C.c_double), ("delta", C.c_double),
                ("gdd", C.c_double), ("seed", C.c_uint64)]


_vp = C.c_void_p
_fp = C.POINTER(C.c_float)
_i = C.c_int
_d = C.c_double

# name -> (restype, argtypes); the authoritative list of exported entry points
SIGNATURES = {
    "cuopo_inputs_default": (None, [C.POINTER(Inputs)]),
    "cuopo_derive_params": (_i, [C.POINTER(Inputs), C.POINTER(Params), C.POINTER(Info)]),
    "cuopo_derive_params_device": (_i, [_vp, _i, _vp, _vp, _vp]),
    "cuopo_sellmeier": (C.c_float, [_i, _i, C.c_float, C.c_float]),
    "cuopo_phase_matching_temp": (C.c_float, [_i, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]),
    "cuopo_make_grids": (_i, [_i, _d, _vp, _vp]),
    "cuopo_linspace": (None, [_vp, C.c_long, C.c_float, C.c_float]),
    "cuopo_pump_cw": (_i, [_vp, _i, _d]),
    "cuopo_pump_ns": (_i, [_vp, _i, _i, _d, _d, _d]),
    "cuopo_noise_host": (_i, [_vp, C.c_long, _d, C.c_uint64, C.c_uint64]),
    "cuopo_noise_device": (_i, [_vp, C.c_long, _d, C.c_uint64, C.c_uint64, _vp]),
    "cuopo_write_dat_real": (_i, [C.c_char_p, _vp, C.c_long]),
    "cuopo_write_dat_complex": (_i, [C.c_char_p, _vp, C.c_long]),
    "cuopo_read_dat_complex": (_i, [C.c_char_p, _vp, C.c_long]),
    "cuopo_plan_create": (_i, [C.POINTER(_vp), C.POINTER(Params), _vp, _vp, _i]),
    "cuopo_plan_destroy": (_i, [_vp]),
    "cuopo_plan_config": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "cuopo_crystal_pass": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "cuopo_round_trips": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, _i, _i, _vp, _d, _vp, _vp]),
    "cuopo_plan_status": (_i, [_vp, C.POINTER(_i), _i]),
    "cuopo_fft_c2c": (_i, [_vp, _vp, _i, _i, _i, _i, _vp]),
    "cuopo_batch_create": (_i, [C.POINTER(_vp), C.POINTER(Params), _vp, _i, _i]),
    "cuopo_batch_create_inputs": (_i, [C.POINTER(_vp), _vp, _vp, _i, _i]),
    "cuopo_batch_destroy": (_i, [_vp]),
    "cuopo_batch_total_elements": (_i, [_vp, C.POINTER(C.c_long)]),
    "cuopo_batch_seed_noise": (_i, [_vp, _d, _vp]),
    "cuopo_batch_set_signal": (_i, [_vp, _vp, _i, _vp]),
    "cuopo_batch_get_signal": (_i, [_vp, _vp, _i, _vp]),
    "cuopo_batch_run": (_i, [_vp, _i, _d, _i, _vp]),
    "cuopo_batch_reset": (_i, [_vp, _vp]),
    "cuopo_batch_step": (_i, [_vp, _i, _i, _d, _i, _vp]),
    "cuopo_batch_pending": (_i, [_vp, C.POINTER(_i), _vp]),
    "cuopo_batch_results": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "cuopo_batch_history": (_i, [_vp, _i, _vp, _i, _vp]),
    "cuopo_batch_wait": (_i, [_vp, _vp]),
    "cuopo_probe_fp32_peak": (_i, [C.POINTER(_d), _vp]),
    "cuopo_probe_fp64_peak": (_i, [C.POINTER(_d), _vp]),
    "cuopo_crystal_pass_noalloc": (_i, [C.POINTER(Params), _vp, _vp, _vp, _vp, _vp]),
    "cuopo_autotune": (_i, [C.POINTER(Params), _i, _i, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_d)]),
    "cuopo_autotune_reset": (_i, []),
    "cuopo_kernel_select": (_i, [_i, _i, _i, _i, _i]),
    "cuopo_kernel_config": (_i, [_i, _i, _i, C.POINTER(_i), C.POINTER(_i)]),
    "cuopo_mlp_create": (_i, [C.POINTER(_vp), _i, _i, _i, _i, _i, C.c_uint64]),
    "cuopo_mlp_destroy": (_i, [_vp]),
    "cuopo_mlp_param_count": (_i, [_vp, C.POINTER(C.c_long)]),
    "cuopo_mlp_set_params": (_i, [_vp, _vp]),
    "cuopo_mlp_get_params": (_i, [_vp, _vp]),
    "cuopo_mlp_forward": (_i, [_vp, _vp, _vp, _i, _vp]),
    "cuopo_mlp_gradients": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _vp]),
    "cuopo_mlp_train_step": (_i, [_vp, _vp, _vp, _i, C.c_float, _vp, _vp]),
    "cuopo_mlp_status": (_i, [_vp]),
    "cuopo_mlp_grad_step": (_i, [_vp, _vp, _vp, _i, _vp, _vp]),
    "cuopo_mlp_grad_buffer": (_i, [_vp, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_long)]),
    "cuopo_mlp_apply_adam": (_i, [_vp, C.c_float, C.c_float, _vp]),
    "cuopo_gemm_bf16": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _vp]),
    "cuopo_fields_from_modes": (_i, [_vp, _i, _i, _i, _d, _vp, _vp]),
    "cuopo_modes_from_spectrum": (_i, [_vp, _i, _i, _i, _d, _vp, _vp]),
    "cuopo_fields_from_bands": (_i, [_vp, _i, _i, _d, _vp, _vp, _vp]),
    "cuopo_sync": (_i, [_vp]),
    "cuopo_last_error": (C.c_char_p, []),
    "cuopo_version": (C.c_char_p, []),
}

_lib = None


def load() -> C.CDLL:
    """Loads the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m cuopo_b200.build` "
                "(the solver has no CPU fallback)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise CuopoError(status, load().cuopo_last_error().decode())
