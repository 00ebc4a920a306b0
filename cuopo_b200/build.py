"""Builds libcuopo_b200.so (and the drop-in CLI) in-tree with nvcc for sm_100a.

Usage: python -m cuopo_b200.build [--force] [--verbose] [--cli-define NS_OPO ...] [--cli-name NAME]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
OBJ = HERE / "_build"
INCLUDE = ROOT / "include"
LIB = HERE / "libcuopo_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I" + str(INCLUDE), "-I" + str(CSRC)]
CC_FLAGS = ["-O2", "-fPIC", "-std=c11", "-Wall", "-Wextra", "-fvisibility=hidden", "-I" + str(INCLUDE),
            "-I" + str(CSRC)]

CU_SOURCES = ["solver.cu", "noise.cu", "fft_api.cu", "probe.cu", "mlp.cu", "params_dev.cu"]
# per-file nvcc flags: the device set-up keeps the host's float rounding (no FMA contraction)
CU_EXTRA = {"params_dev.cu": ["-fmad=false"]}
C_SOURCES = ["params.c", "dat_io.c"]
BIN = HERE / "bin"
CLI = BIN / "cuopo"


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _cc() -> str:
    return shutil.which("gcc") or "cc"


def _deps(src: Path) -> list[Path]:
    return [src] + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "cuopo.h", Path(__file__)]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-3:]}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles every CUDA/C source of the library for sm_100a and links the .so."""
    OBJ.mkdir(exist_ok=True)
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = CSRC / s
        obj = OBJ / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, _deps(src)):
            cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, *CU_EXTRA.get(s, []), "-c", str(src), "-o", str(obj)]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for s in C_SOURCES:
        src = CSRC / s
        obj = OBJ / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, _deps(src)):
            jobs.append([_cc(), *CC_FLAGS, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        list(ex.map(lambda c: _run(c, verbose or ptxas_verbose), jobs))
    if force or jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([_nvcc(), *ARCH, "-shared", "--cudart", "static", "-o", str(tmp), *map(str, objs), "-lm"], verbose)
        os.replace(tmp, LIB)
    return LIB


def _cuda_home() -> Path:
    return Path(_nvcc()).resolve().parent.parent


def build_cli(defines: tuple[str, ...] = (), name: str = "cuopo", force: bool = False, verbose: bool = False) -> Path:
    """Builds the drop-in executable (csrc/cli.cpp) against the library.

    defines: the reference's compile-time switches (CW_OPO / NS_OPO,
    THREE_EQS, PPLN / SPPLT, SIZE=, NZ=, NRT=) that set the executable's
    defaults; run-time options override them."""
    lib = build(force=force, verbose=verbose)
    BIN.mkdir(exist_ok=True)
    out = BIN / name
    src = CSRC / "cli.cpp"
    if not force and not _stale(out, [src, lib, INCLUDE / "cuopo.h", Path(__file__)]):
        return out
    cuda = _cuda_home()
    tmp = out.with_name(out.name + ".tmp")
    _run(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", *[f"-D{d}" for d in defines], "-I" + str(INCLUDE),
          "-I" + str(cuda / "include"), str(src), "-o", str(tmp), "-L" + str(HERE), "-lcuopo_b200",
          "-Wl,-rpath,$ORIGIN/..", "-L" + str(cuda / "lib64"), "-lcudart_static", "-ldl", "-lpthread", "-lrt"],
         verbose)
    os.replace(tmp, out)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/spill use (-Xptxas -v)")
    ap.add_argument("--cli-define", action="append", default=[],
                    help="build the drop-in executable with this -D switch (repeatable, e.g. NS_OPO, THREE_EQS)")
    ap.add_argument("--cli-name", default="cuopo", help="name of the executable under cuopo_b200/bin")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))
    print(build_cli(tuple(a.cli_define), a.cli_name, force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
