"""Builds libcuopo_b200.so (and the drop-in CLI) in-tree with nvcc for sm_100a.

Usage: python -m cuopo_b200.build [--force] [--verbose]
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

CU_SOURCES = ["solver.cu", "noise.cu", "fft_api.cu", "probe.cu"]
C_SOURCES = ["params.c", "dat_io.c"]


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
            cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
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


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/spill use (-Xptxas -v)")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))


if __name__ == "__main__":
    main()
