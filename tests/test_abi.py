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


def test_new_entry_points_reject_bad_arguments_before_touching_the_gpu():
    """Argument checks of the warm-start and device set-up entry points run
    before any CUDA call, so they answer CUOPO_EINVAL on a machine without a
    GPU as well."""
    import ctypes as C
    lib = cu.load()
    h = C.c_void_p()
    # MLP: n_in > 64, width not a multiple of 128, depth 0
    assert lib.cuopo_mlp_create(C.byref(h), 65, 512, 4, 512, 4096, 0) == cu.EINVAL
    assert lib.cuopo_mlp_create(C.byref(h), 4, 500, 4, 512, 4096, 0) == cu.EINVAL
    assert lib.cuopo_mlp_create(C.byref(h), 4, 512, 0, 512, 4096, 0) == cu.EINVAL
    assert lib.cuopo_mlp_create(None, 4, 512, 4, 512, 4096, 0) == cu.EINVAL
    # GEMM: NULL operands, M not a multiple of 128
    assert lib.cuopo_gemm_bf16(None, None, None, 128, 64, 64, 1, 0, None, None) == cu.EINVAL
    buf = (C.c_float * 16)()
    assert lib.cuopo_gemm_bf16(buf, buf, buf, 100, 64, 64, 1, 0, None, None) == cu.EINVAL
    # field synthesis: n_t not a power of 2 / too small, n_modes not a multiple of 16
    assert lib.cuopo_fields_from_bands(buf, 1, 100, 1.0, buf, None, None) == cu.EINVAL
    assert lib.cuopo_fields_from_modes(buf, 1, 20, 1024, 1.0, buf, None) == cu.EINVAL
    # one grid row per instance: at most 65535 per call
    assert lib.cuopo_fields_from_bands(buf, 65536, 1024, 1.0, buf, None, None) == cu.EINVAL
    assert lib.cuopo_fields_from_modes(buf, 65536, 256, 1024, 1.0, buf, None) == cu.EINVAL
    assert lib.cuopo_modes_from_spectrum(buf, 1, 1024, 48, 1.0, buf, None) == cu.EINVAL
    # device set-up: NULL arrays, no instances
    assert lib.cuopo_derive_params_device(None, 4, None, None, None) == cu.EINVAL
    assert lib.cuopo_derive_params_device(buf, 0, buf, buf, None) == cu.EINVAL
    # data-parallel pieces on a NULL network
    assert lib.cuopo_mlp_apply_adam(None, 1e-3, 1.0, None) == cu.EINVAL
    assert lib.cuopo_mlp_grad_buffer(None, None, None) == cu.EINVAL
