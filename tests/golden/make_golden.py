"""Generates the golden vectors in tests/golden/ by running the reference's own
crystal-pass and cavity kernels with cuFFT (oracle/_ref, built from the
reference's sources by oracle/build_ref.sh) on seeded inputs.

Needs a GPU.  Usage: python tests/golden/make_golden.py [outdir]
Each case is saved as <name>.npz with the cuopo_params fields (p_<name>),
the inputs (Ap0, As0, Ai0, pump, w, T) and the reference's outputs after the
run (Ap, As, Ai, saved round trips sv_p/sv_s/sv_i, ps_hist).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import cuopo_b200 as cu  # noqa: E402
from oracle import binding as ob  # noqa: E402
from tests.helpers import params_2eq, params_3eq, random_field  # noqa: E402

CASES = {
    # name: (crystal, params, n_rt, rts to run, save window)
    "ppln_cw_2eq_1024": ("ppln", lambda: params_2eq(n_t=1024, n_z=8, delta=0.05, gdd_percent=50.0, use_eom=1),
                         4, 4, (1, 3)),
    "ppln_pass_2eq_256": ("ppln", lambda: params_2eq(n_t=256, n_z=10), 1, 1, (0, 1)),
    "spplt_ns_3eq_1024": ("spplt", lambda: params_3eq(n_t=1024, n_z=8, gdd_percent=30.0, delta=-0.04), 6, 6, (0, 6)),
}


def make(name, outdir: Path):
    crystal, mk, n_rt, count, (sf, sc) = CASES[name]
    p = mk()
    n = p.n_t
    T, w = cu.make_grids(n, p.t_rt)
    Ap0 = random_field(n, 0.08, 11).astype(np.complex64)
    As0 = random_field(n, 0.3, 12).astype(np.complex64)
    Ai0 = random_field(n, 0.3, 13).astype(np.complex64) if p.n_eqs == 3 else np.zeros(0, np.complex64)
    if p.regime == cu.NS:
        pump = cu.pump_ns(n, n_rt, p.t_rt, p.ap0 * 3, 2.0 * p.t_rt)
    else:
        pump = np.full(n, p.ap0 * 3, np.complex64)
    A = [Ap0.copy(), As0.copy(), Ai0.copy() if p.n_eqs == 3 else None]
    sv = [np.zeros(n * sc, np.complex64) for _ in range(3)]
    ps = np.zeros(count)
    ob.ref_round_trips(crystal, p, w, T, A[0], A[1], A[2], pump, n_rt, 0, count, sv[0], sv[1],
                       sv[2] if p.n_eqs == 3 else None, sf, sc, ps)
    fields = {f"p_{k}": v for k, v in p.to_dict().items()}
    np.savez_compressed(outdir / f"{name}.npz", **fields, crystal=crystal, n_rt=n_rt, count=count, save_first=sf,
                        save_count=sc, Ap0=Ap0, As0=As0, Ai0=Ai0, pump=pump, w=w, T=T, Ap=A[0], As=A[1],
                        Ai=A[2] if p.n_eqs == 3 else np.zeros(0, np.complex64), sv_p=sv[0], sv_s=sv[1],
                        sv_i=sv[2] if p.n_eqs == 3 else np.zeros(0, np.complex64), ps_hist=ps)
    print("wrote", outdir / f"{name}.npz")


if __name__ == "__main__":
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    out.mkdir(parents=True, exist_ok=True)
    for name in CASES:
        make(name, out)
