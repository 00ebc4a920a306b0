"""The drop-in executable cuopo_b200/bin/cuopo (csrc/cli.cpp): the reference's
12 positional arguments (src/cuOPO.sh:159, src/cuOPO.cu:92-267) and its
output files (src/cuOPO.cu:273-286,620-635; files.cuh:21-62).

CPU tests run the executable with --setup-only (no GPU call): argument
errors, the written inputs and grids against the library's host set-up,
which tests/test_params.py pins bit for bit to the reference's host code.
The GPU tests run whole simulations and compare the saved round trips with
the FP64 oracle started from the same input files.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import cuopo_b200 as cu
from cuopo_b200 import build as cb

ARGS_2EQ = ["532", "27", "6.970206862971646", "4", "98", "0.05", "50", "0", "0", "0.6", "4", "5"]
ARGS_3EQ = ["532", "27", "8.719670871908674", "3", "98", "-0.04", "30", "0", "0", "0", "0", "20"]


@pytest.fixture(scope="module")
def exe() -> Path:
    return cb.build_cli()


def run(exe, args, cwd, check=True):
    r = subprocess.run([str(exe), *args], cwd=cwd, capture_output=True, text=True, timeout=600)
    if check and r.returncode != 0:
        raise AssertionError(f"cuopo exited {r.returncode}: {r.stderr}")
    return r


def read_real(path: Path) -> np.ndarray:
    return np.loadtxt(path, dtype=np.float64).astype(np.float32)


def read_complex(prefix: Path) -> np.ndarray:
    return read_real(Path(str(prefix) + "_r.dat")) + 1j * read_real(Path(str(prefix) + "_i.dat"))


def test_usage_errors(exe, tmp_path):
    assert run(exe, ["--help"], tmp_path, check=False).returncode == 2
    r = run(exe, ["--setup-only", *ARGS_2EQ[:11]], tmp_path, check=False)
    assert r.returncode == 2 and "12 positional" in r.stderr
    r = run(exe, ["--setup-only", *ARGS_2EQ[:3], "four", *ARGS_2EQ[4:]], tmp_path, check=False)
    assert r.returncode == 2 and "not a number" in r.stderr
    r = run(exe, ["--bogus", *ARGS_2EQ], tmp_path, check=False)
    assert r.returncode == 2 and "unknown option" in r.stderr
    r = run(exe, ["--setup-only", "--n-t", "1000", *ARGS_2EQ], tmp_path, check=False)
    assert r.returncode == 1 and "power of 2" in r.stderr


def setup_params(n_t, n_z, n_rt, args, **kw):
    inp = cu.default_inputs(n_t=n_t, n_z=n_z, n_rt=n_rt, lp_nm=float(args[0]), temp_c=float(args[1]),
                            lambda_um=float(args[2]), n_thr=float(args[3]), r_percent=float(args[4]),
                            delta=float(args[5]), gdd_percent=float(args[6]), tod_percent=float(args[7]),
                            use_eom=int(args[8]), mod_depth_pi=float(args[9]), freq_det_mhz=float(args[10]),
                            lcr_mm=float(args[11]), **kw)
    return cu.derive_params(inp)[0], inp


def test_setup_files_cw(exe, tmp_path):
    n_t, n_rt = 256, 70
    run(exe, ["--setup-only", "--quiet", "--n-t", str(n_t), "--n-z", "4", "--n-rt", str(n_rt), "--seed", "7",
              *ARGS_2EQ], tmp_path)
    p, _ = setup_params(n_t, 4, n_rt, ARGS_2EQ)
    T, _ = cu.make_grids(n_t, p.t_rt)
    assert np.array_equal(read_real(tmp_path / "T.dat"), T)
    # CW: the saved window is the last 64 round trips (cuOPO.cu:154-166)
    t_width = np.float32(p.t_rt) * np.float32(64)
    Tp = cu.linspace(n_t * 64, float(np.float32(-0.5 * float(t_width))), float(np.float32(0.5 * float(t_width))))
    assert np.array_equal(read_real(tmp_path / "Tp.dat"), Tp)
    assert read_real(tmp_path / "freq.dat").shape == (n_t * 64,)
    assert np.array_equal(read_complex(tmp_path / "pump_input"), cu.pump_cw(n_t, p.ap0))
    assert np.array_equal(read_complex(tmp_path / "signal_input"), cu.noise_host(n_t, 1e-15, 7, 1))
    assert not (tmp_path / "idler_input_r.dat").exists()
    assert not (tmp_path / "signal_output_r.dat").exists()


def test_setup_files_ns_three_eqs(exe, tmp_path):
    n_t, n_rt = 128, 5
    run(exe, ["--setup-only", "--quiet", "--ns", "--three-eqs", "--spplt", "--ls-nm", "1550", "--n-t", str(n_t),
              "--n-z", "4", "--n-rt", str(n_rt), "--seed", "11", *ARGS_3EQ], tmp_path)
    p, inp = setup_params(n_t, 4, n_rt, ARGS_3EQ, crystal=cu.SPPLT, n_eqs=3, regime=cu.NS, ls_nm=1550.0)
    assert p.n_eqs == 3 and p.regime == cu.NS
    assert np.array_equal(read_complex(tmp_path / "pump_input"), cu.pump_ns(n_t, n_rt, p.t_rt, p.ap0, inp.fwhm_ps))
    assert np.array_equal(read_complex(tmp_path / "idler_input"), cu.noise_host(n_t, 1e-15, 11, 2))
    assert read_real(tmp_path / "Tp.dat").shape == (n_t * n_rt,)


def test_binary_format(exe, tmp_path):
    n_t = 64
    run(exe, ["--setup-only", "--quiet", "--format", "bin", "--n-t", str(n_t), "--n-rt", "3", "--seed", "2",
              *ARGS_2EQ], tmp_path)
    s = np.fromfile(tmp_path / "signal_input.c64", dtype=np.complex64)
    assert np.array_equal(s, cu.noise_host(n_t, 1e-15, 2, 1))
    assert np.fromfile(tmp_path / "T.f32", dtype=np.float32).shape == (n_t,)


def test_signal_input_is_read_back(exe, tmp_path):
    n_t = 64
    v = (np.arange(n_t) * 1e-3 - 1j * np.arange(n_t) * 2e-3).astype(np.complex64)
    cu.write_dat_complex(str(tmp_path / "given"), v)
    run(exe, ["--setup-only", "--quiet", "--n-t", str(n_t), "--n-rt", "3", "--signal-input",
              str(tmp_path / "given"), *ARGS_2EQ], tmp_path)
    assert np.array_equal(read_complex(tmp_path / "signal_input"), v)


# ------------------------------------------------------------------ GPU runs

def oracle_saves(p, n_rt, save_first, save_count, pump, As0, Ai0=None):
    from oracle import binding as ob
    T, w = cu.make_grids(p.n_t, p.t_rt)
    n = p.n_t
    A = [np.zeros(n, np.complex128), As0.astype(np.complex128),
         Ai0.astype(np.complex128) if Ai0 is not None else None]
    sv = [np.zeros(n * save_count, np.complex128) for _ in range(3)]
    ps = np.zeros(n_rt)
    ob.round_trips(p, w.astype(np.float64), T.astype(np.float64), A[0], A[1], A[2], pump.astype(np.complex128),
                   n_rt, 0, n_rt, sv[0], sv[1], sv[2] if Ai0 is not None else None, save_first, save_count, ps)
    return sv


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.gpu
def test_cli_cw_run_matches_oracle(exe, tmp_path):
    """CW 2-eq with GDD, detuning and the modulator: the last 64 of 70 round
    trips saved, FP32 run vs FP64 oracle from the same inputs (5e-5)."""
    n_t, n_z, n_rt = 1024, 8, 70
    args = list(ARGS_2EQ)
    args[8] = "1"  # modulator on
    run(exe, ["--quiet", "--n-t", str(n_t), "--n-z", str(n_z), "--n-rt", str(n_rt), "--seed", "5", *args], tmp_path)
    p, _ = setup_params(n_t, n_z, n_rt, args)
    pump = read_complex(tmp_path / "pump_input")
    As0 = read_complex(tmp_path / "signal_input")
    sv = oracle_saves(p, n_rt, n_rt - 64, 64, pump, As0)
    assert rel_l2(read_complex(tmp_path / "signal_output"), sv[1]) < 5e-5
    assert rel_l2(read_complex(tmp_path / "pump_output"), sv[0]) < 5e-5


@pytest.mark.gpu
def test_cli_ns_three_eqs_run_matches_oracle(exe, tmp_path):
    """NS 3-eq sPPLT: every round trip saved (cuOPO.cu:599-608)."""
    n_t, n_z, n_rt = 1024, 8, 6
    run(exe, ["--quiet", "--ns", "--three-eqs", "--spplt", "--ls-nm", "1550", "--n-t", str(n_t), "--n-z", str(n_z),
              "--n-rt", str(n_rt), "--seed", "9", *ARGS_3EQ], tmp_path)
    p, _ = setup_params(n_t, n_z, n_rt, ARGS_3EQ, crystal=cu.SPPLT, n_eqs=3, regime=cu.NS, ls_nm=1550.0)
    pump = read_complex(tmp_path / "pump_input")
    sv = oracle_saves(p, n_rt, 0, n_rt, pump, read_complex(tmp_path / "signal_input"),
                      read_complex(tmp_path / "idler_input"))
    for name, ref in (("pump_output", sv[0]), ("signal_output", sv[1]), ("idler_output", sv[2])):
        assert rel_l2(read_complex(tmp_path / name), ref) < 5e-5, name


@pytest.mark.gpu
def test_cli_f64_binary_run_matches_oracle(exe, tmp_path):
    """--f64 --format bin: FP64 fields through the executable, raw complex64
    outputs of the saved round trips against the FP64 oracle (the outputs
    are written as float pairs, so the bound is float rounding: 1e-6)."""
    n_t, n_z, n_rt = 512, 6, 66
    run(exe, ["--quiet", "--f64", "--format", "bin", "--n-t", str(n_t), "--n-z", str(n_z), "--n-rt", str(n_rt),
              "--seed", "3", *ARGS_2EQ], tmp_path)
    p, _ = setup_params(n_t, n_z, n_rt, ARGS_2EQ)
    pump = np.fromfile(tmp_path / "pump_input.c64", dtype=np.complex64)
    As0 = np.fromfile(tmp_path / "signal_input.c64", dtype=np.complex64)
    sv = oracle_saves(p, n_rt, n_rt - 64, 64, pump, As0)
    got = np.fromfile(tmp_path / "signal_output.c64", dtype=np.complex64)
    assert got.shape == (64 * n_t,)
    assert rel_l2(got, sv[1]) < 1e-6
