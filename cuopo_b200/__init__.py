"""cuopo_b200: a B200 (sm_100a) split-step Fourier coupled-wave OPO solver.

A drop-in for the crystal pass and cavity round-trip loop of cuOPO.  The
solver lives in libcuopo_b200.so (C ABI: include/cuopo.h); this package
binds it with ctypes.
"""
from ._lib import (CW, EINVAL, ENOMEM, ENONFINITE, EUNSUPPORTED, F32, F32_PHASE32, F64, NS, OK, PPLN, SPPLT, CuopoError,
                   Info, Inputs, Params, load)
from .api import (Batch, Plan, autotune, autotune_reset, default_inputs, derive_params, derive_params_device, fft_c2c, kernel_config, kernel_select,
                  linspace,
                  make_grids, noise_device, noise_host,
                  phase_matching_temp, probe_fp32_peak, probe_fp64_peak, pump_cw, pump_ns, read_dat_complex, sellmeier, sync, write_dat_complex,
                  write_dat_real)

__all__ = [
    "CW", "NS", "PPLN", "SPPLT", "F32", "F32_PHASE32", "F64", "OK", "EINVAL", "ENOMEM", "ENONFINITE", "EUNSUPPORTED",
    "Batch", "CuopoError", "autotune", "autotune_reset", "kernel_config", "kernel_select", "Info", "Inputs", "Params", "Plan", "default_inputs", "derive_params", "derive_params_device", "fft_c2c", "linspace",
    "make_grids", "noise_device", "noise_host", "phase_matching_temp", "probe_fp32_peak", "probe_fp64_peak", "pump_cw", "pump_ns",
    "read_dat_complex", "sellmeier", "sync", "write_dat_complex", "write_dat_real", "load",
]
