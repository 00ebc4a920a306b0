"""Batched parameter derivation on the device (cuopo_derive_params_device)
against the host's cuopo_derive_params, which is bit-exact with the
reference's own set-up (tests/test_params.py).  Float operations round the
same on both sides (the device file is compiled without FMA contraction);
CUDA's powf/pow may round differently from glibc's in the last bits, and a
few ulps of the refractive indices move the phase mismatch dk, a float
difference with cancellation (cuOPO.cu:122-126), by ~1e-6 per um.  Bounds:
relative 1e-5 per derived value except dk, absolute 3e-5 per um for dk
(measured on the B200: 755 of 1024 instances bit-identical, at most 1.5e-6
relative (GVD), dk within 3.0e-6 per um; the per-field maxima are
printed)."""
import time

import numpy as np
import pytest

import cuopo_b200 as cu

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FIELDS = ("vp", "vs", "vi", "b2p", "b2s", "b2i", "dk", "kp", "ks", "ki", "dz", "Rs", "Ri", "delta", "gdd",
          "mod_depth", "fpm", "t_rt", "ap0")


def _inputs(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        three = k % 3 == 0
        spplt = k % 2 == 0
        inp = cu.default_inputs(crystal=cu.SPPLT if spplt else cu.PPLN, n_eqs=3 if three else 2,
                                regime=cu.NS if three else cu.CW, n_t=int(2 ** rng.integers(10, 16)),
                                n_z=int(rng.integers(20, 400)), lp_nm=float(rng.uniform(520, 540)),
                                ls_nm=float(rng.uniform(1400, 1700)) if three else 0.0,
                                lambda_um=float((8.72 if spplt else 6.97) + rng.uniform(-0.3, 0.3)),
                                n_thr=float(rng.uniform(1.1, 6)), r_percent=float(rng.uniform(80, 99.5)),
                                delta=float(rng.uniform(-1, 1)), gdd_percent=float(rng.uniform(-100, 100)),
                                lcr_mm=float(rng.uniform(2, 30)), use_eom=int(rng.integers(0, 2)),
                                mod_depth_pi=float(rng.uniform(0.1, 1)), freq_det_mhz=float(rng.uniform(0, 10)))
        if k % 7 == 0:
            # the argv[2] temperature instead of the scan
            inp.temp_from_scan = 0
            inp.temp_c = float(rng.uniform(20, 120))
        out.append(inp)
    return out


def test_device_setup_matches_host():
    inputs = _inputs(1024, 5)
    t0 = time.perf_counter()
    host = [cu.derive_params(x)[0] for x in inputs]
    t_host = time.perf_counter() - t0
    cu.derive_params_device(inputs[:8])          # first launch (module load) out of the timing
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dev = cu.derive_params_device(inputs)
    t_dev = time.perf_counter() - t0
    rel = {f: 0.0 for f in FIELDS}
    same = 0
    for h, d in zip(host, dev):
        for f in FIELDS:
            a, b = getattr(h, f), getattr(d, f)
            if a != b:
                rel[f] = max(rel[f], abs(a - b) if f == "dk" else abs(a - b) / max(abs(a), 1e-300))
        same += all(getattr(h, f) == getattr(d, f) for f in FIELDS)
    print(f"1024 instances: host {t_host * 1e3:.0f} ms, device {t_dev * 1e3:.1f} ms (incl. copies); "
          f"bit-identical {same}; largest differences", {f: f"{v:.1e}" for f, v in rel.items() if v})
    assert rel.pop("dk") <= 3e-5
    assert max(rel.values()) <= 1e-5


def test_device_setup_rejects_invalid_instances():
    inputs = _inputs(4, 6)
    inputs[2].n_t = 1000
    with pytest.raises(cu.CuopoError) as e:
        cu.derive_params_device(inputs)
    assert e.value.status == cu.EINVAL and "instance 2" in str(e.value)
