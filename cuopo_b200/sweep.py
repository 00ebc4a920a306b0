"""Parameter sweeps as batches.

The reference explores parameter space with nested shell loops that run one
process per point (src/cuOPO.sh:91-174).  Here a sweep is a list of
cuopo_instance records solved together by cuopo_batch_run.
"""
from __future__ import annotations

import numpy as np

from . import api
from ._lib import CW, PPLN


def cw_base_inputs(n_t: int = 8192, n_z: int = 100, **kw):
    """CW 2-equation MgO:PPLN cavity: 532 nm pump, degenerate 1064 nm signal,
    5 mm crystal, QPM period for dk = 0 at 26.85 C (the scan then picks 26.859 C)."""
    args = dict(crystal=PPLN, n_eqs=2, regime=CW, n_t=n_t, n_z=n_z, n_rt=5000, lp_nm=532.0,
                lambda_um=6.970206862971646, n_thr=4.0, r_percent=98.0, lcr_mm=5.0)
    args.update(kw)
    return api.default_inputs(**args)


def random_cw_sweep(count: int = 1024, rng_seed: int = 0, n_t_choices=(4096, 8192, 16384, 32768),
                    n_thr=(1.2, 6.0), delta_rad=(-np.pi, np.pi), gdd_fs2=(-500.0, 500.0), refl=(0.90, 0.99),
                    n_z: int = 100):
    """Uniformly drawn CW sweep: pump ratio N, detuning delta [rad], intracavity
    GDD [fs^2], reflectivity R and grid size; instance k's noise seed is k.

    Returns (base params, list of instance dicts, table of the drawn values)."""
    rng = np.random.default_rng(rng_seed)
    N = rng.uniform(*n_thr, count)
    dl = rng.uniform(*delta_rad, count)
    gd = rng.uniform(*gdd_fs2, count)
    R = rng.uniform(*refl, count)
    nt = rng.choice(np.asarray(n_t_choices), count)
    base, _ = api.derive_params(cw_base_inputs(n_t=int(nt[0]), n_z=n_z))
    insts = []
    for k in range(count):
        # the pump amplitude follows the threshold of each (N, R) point (cuOPO.cu:222-229)
        p, _ = api.derive_params(cw_base_inputs(n_t=int(nt[k]), n_z=n_z, n_thr=float(N[k]),
                                                r_percent=float(R[k]) * 100.0))
        insts.append(dict(n_t=int(nt[k]), ap0=p.ap0, Rs=p.Rs, delta=float(dl[k]) / np.pi,
                          gdd=float(gd[k]) * 1e-6, seed=k))
    table = dict(n_thr=N, delta_rad=dl, gdd_fs2=gd, refl=R, n_t=nt)
    return base, insts, table


def growth_estimate(table, noise_sigma: float = 1e-15) -> np.ndarray:
    """Rough round trips from noise to saturation, ln(P_sat/P_0) / (2 (sqrt(N)-1)(1-R));
    used only to order work (longest first)."""
    g = 2.0 * (np.sqrt(table["n_thr"]) - 1.0) * (1.0 - table["refl"])
    return np.log(0.2 / (2 * noise_sigma ** 2)) / np.maximum(g, 1e-6)


def script_sweep(base: "api.Inputs | None" = None, **axes) -> list:
    """The nested loops of the reference's sweep script (src/cuOPO.sh:91-174)
    as a list of per-instance inputs: the Cartesian product of the given
    axes over any cuopo_inputs fields (lp_nm, lambda_um, n_thr, r_percent,
    delta, gdd_percent, tod_percent, use_eom, mod_depth_pi, freq_det_mhz,
    lcr_mm, n_t, n_z, n_eqs, ...), the first axis outermost.  Run them with
    api.Batch(None, inputs)."""
    import ctypes
    import itertools
    base = base if base is not None else cw_base_inputs()
    names = list(axes)
    out = []
    for vals in itertools.product(*(axes[n] for n in names)):
        inp = api.Inputs()
        ctypes.pointer(inp)[0] = base
        for n, v in zip(names, vals):
            setattr(inp, n, v)
        out.append(inp)
    return out
