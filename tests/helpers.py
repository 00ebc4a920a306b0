"""Shared set-up for the tests: parameter sets, fields and error norms."""
from __future__ import annotations

import numpy as np

import cuopo_b200 as cu


def params_2eq(n_t=1024, n_z=8, n_thr=4.0, r_percent=98.0, delta=0.0, gdd_percent=0.0, lcr_mm=5.0,
               use_eom=0, regime=cu.CW, **kw):
    """MgO:PPLN, 532 nm pump, degenerate signal (the C1 physics at a small grid)."""
    inp = cu.default_inputs(crystal=cu.PPLN, n_eqs=2, regime=regime, n_t=n_t, n_z=n_z, n_rt=100, lp_nm=532.0,
                            lambda_um=6.970206862971646, n_thr=n_thr, r_percent=r_percent, delta=delta,
                            gdd_percent=gdd_percent, lcr_mm=lcr_mm, use_eom=use_eom, mod_depth_pi=0.6,
                            freq_det_mhz=4.0, **kw)
    return cu.derive_params(inp)[0]


def params_3eq(n_t=1024, n_z=8, n_thr=3.0, r_percent=98.0, delta=0.0, gdd_percent=0.0, lcr_mm=20.0,
               regime=cu.NS, n_rt=16, **kw):
    """MgO:sPPLT, 532 nm pump, 1550 nm signal (the C2 physics at a small grid)."""
    inp = cu.default_inputs(crystal=cu.SPPLT, n_eqs=3, regime=regime, n_t=n_t, n_z=n_z, n_rt=n_rt, lp_nm=532.0,
                            ls_nm=1550.0, lambda_um=8.719670871908674, n_thr=n_thr, r_percent=r_percent, delta=delta,
                            gdd_percent=gdd_percent, lcr_mm=lcr_mm, **kw)
    return cu.derive_params(inp)[0]


def random_field(n, scale, seed):
    rng = np.random.default_rng(seed)
    return (scale * (rng.standard_normal(n) + 1j * rng.standard_normal(n))).astype(np.complex128)


def rel_l2(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
