"""The allocation-free crystal pass (cuopo_crystal_pass_noalloc).

Some callers cannot call cudaMalloc -- a plugin inside a process whose
device memory belongs to another allocator or a fixed budget.  This entry
point keeps its tables in a fixed device array inside the library instead.
It is checked here, through the C ABI, against the plan-based
cuopo_crystal_pass on the same inputs (FP32 tolerance 5e-6 relative L2, the
pass tolerance of the other GPU tests), for two passes in a row, with the
frequency grid given and built inside the call, and for its size limits.
The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import cuopo_b200 as cu
from cuopo_b200 import _lib
from tests.helpers import params_2eq, params_3eq, random_field, rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _noalloc(p, w, Ap, As, Ai):
    lib = cu.load()
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.cuopo_crystal_pass_noalloc(C.byref(p), None if w is None else w.ctypes.data, Ap.data_ptr(),
                                              As.data_ptr(), None if Ai is None else Ai.data_ptr(), stream))


@pytest.mark.parametrize("neq,n_t,grid_inside", [(2, 2048, False), (2, 8192, False), (3, 1024, False),
                                                 (3, 4096, False), (3, 8192, False), (2, 2048, True),
                                                 (3, 1024, True)])
def test_noalloc_pass_matches_plan_pass_twice(neq, n_t, grid_inside):
    p = params_2eq(n_t=n_t, n_z=12) if neq == 2 else params_3eq(n_t=n_t, n_z=12)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    init = [random_field(n_t, 0.08, 1), random_field(n_t, 0.3, 2)] + ([random_field(n_t, 0.3, 3)] if neq == 3 else [])
    a = [torch.from_numpy(x.astype(np.complex64)).cuda() for x in init]
    b = [x.clone() for x in a]
    c = [x.clone() for x in a]
    with cu.Plan(p, w, T, precision=cu.F32) as plan:
        for _ in range(2):
            plan.crystal_pass(*a, *([None] if neq == 2 else []))
            _noalloc(p, w, b[0], b[1], b[2] if neq == 3 else None)
            if grid_inside:
                _noalloc(p, None, c[0], c[1], c[2] if neq == 3 else None)
            torch.cuda.synchronize()
            for x, y, z in zip(a, b, c):
                assert rel_l2(y.cpu().numpy(), x.cpu().numpy()) < 5e-6
                if grid_inside:
                    # the grid built inside the call is cuopo_make_grids' grid bit for bit
                    assert torch.equal(y, z)


def test_noalloc_rejects_sizes_beyond_its_array():
    p = params_2eq(n_t=16384, n_z=4)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    x = torch.zeros(p.n_t, dtype=torch.complex64, device="cuda")
    with pytest.raises(cu.CuopoError) as e:
        _noalloc(p, w, x, x.clone(), None)
    assert e.value.status == cu.EINVAL and "384 KiB" in str(e.value)
    p = params_2eq(n_t=1024, n_z=2000)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    x = torch.zeros(p.n_t, dtype=torch.complex64, device="cuda")
    with pytest.raises(cu.CuopoError) as e:
        _noalloc(p, w, x, x.clone(), None)
    assert e.value.status == cu.EINVAL
