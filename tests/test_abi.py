"""The C-ABI library loads and exports every entry point include/cuopo.h declares (no GPU needed)."""
import re
from pathlib import Path

import cuopo_b200 as cu
from cuopo_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / "include" / "cuopo.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cuopo_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cuopo_crystal_pass" in names and "cuopo_round_trips" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = cu.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES), set(declared_functions()) - set(_lib.SIGNATURES)


def test_version_and_errors():
    lib = cu.load()
    assert b"sm_100a" in lib.cuopo_version()
    p = cu.Params()
    p.n_eqs = 5
    try:
        cu.Plan(p)
    except cu.CuopoError as e:
        assert e.status == cu.EINVAL
        assert "n_eqs" in str(e)
    else:
        raise AssertionError("invalid n_eqs accepted")
