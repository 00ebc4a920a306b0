"""Pins the FP64 CPU oracle to the reference's own output (no GPU needed).

The golden vectors (tests/golden/*.npz, made by tests/golden/make_golden.py)
come from the reference's crystal-pass and cavity kernels with cuFFT, in
float, on seeded inputs.  The oracle reruns the same inputs in double; the
two differ by the reference's float rounding only, so the bar is a relative
L2 of 5e-4 per field and 5e-4 on the per-round-trip signal power -- far
below the O(1) differences a wrong quirk, sign or ordering would produce.
"""
from pathlib import Path

import numpy as np
import pytest

import cuopo_b200 as cu
from oracle import binding as ob
from tests.helpers import rel_l2

GOLDEN = Path(__file__).resolve().parent / "golden"
FILES = sorted(GOLDEN.glob("*.npz"))


def load_params(d):
    p = cu.Params()
    for k, _ in cu.Params._fields_:
        setattr(p, k, d["p_" + k].item())
    return p


@pytest.mark.skipif(not FILES, reason="no golden vectors committed")
@pytest.mark.parametrize("path", FILES, ids=[f.stem for f in FILES])
def test_oracle_matches_reference_golden(path):
    d = np.load(path, allow_pickle=False)
    p = load_params(d)
    n = p.n_t
    three = p.n_eqs == 3
    A = [d["Ap0"].astype(np.complex128), d["As0"].astype(np.complex128),
         d["Ai0"].astype(np.complex128) if three else None]
    sf, sc, count = int(d["save_first"]), int(d["save_count"]), int(d["count"])
    sv = [np.zeros(n * sc, np.complex128) for _ in range(3)]
    ps = np.zeros(count)
    ob.round_trips(p, d["w"].astype(np.float64), d["T"].astype(np.float64), A[0], A[1], A[2],
                   d["pump"].astype(np.complex128), int(d["n_rt"]), 0, count, sv[0], sv[1],
                   sv[2] if three else None, sf, sc, ps)
    assert rel_l2(A[0], d["Ap"]) < 5e-4
    assert rel_l2(A[1], d["As"]) < 5e-4
    if three:
        assert rel_l2(A[2], d["Ai"]) < 5e-4
        assert rel_l2(sv[2], d["sv_i"]) < 5e-4
    assert rel_l2(sv[0], d["sv_p"]) < 5e-4
    assert rel_l2(sv[1], d["sv_s"]) < 5e-4
    assert np.max(np.abs(ps - d["ps_hist"]) / d["ps_hist"]) < 5e-4


def test_golden_inputs_use_reference_grids():
    """The golden grids are the reference's float linspace/fftshift grids."""
    for path in FILES:
        d = np.load(path, allow_pickle=False)
        T, w = cu.make_grids(int(d["p_n_t"]), float(d["p_t_rt"]))
        assert np.array_equal(T, d["T"]) and np.array_equal(w, d["w"])
