"""Physics checks of the GPU solver that need no reference run: the
degenerate DRO's steady-state signal power scales as sqrt(N) - 1 with the
pump ratio N (plane-wave theory, non-resonant pump), and the FP32 steady
state agrees with the FP64 CPU oracle's from the same start."""
import numpy as np
import pytest

import cuopo_b200 as cu
from oracle import binding as ob
from tests.helpers import params_2eq

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def gpu_steady(n_thr, n_t=512, n_z=10, max_rt=20000, tol=1e-7):
    p = params_2eq(n_t=n_t, n_z=n_z, n_thr=n_thr, r_percent=98.0)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    with cu.Plan(p, w, T, precision=cu.F32) as plan:
        Ap = torch.zeros(n_t, dtype=torch.complex64, device="cuda")
        As = torch.full((n_t,), 1e-2, dtype=torch.complex64, device="cuda")
        pump = torch.full((n_t,), complex(np.float32(p.ap0)), dtype=torch.complex64, device="cuda")
        hist = torch.zeros(max_rt, dtype=torch.float64, device="cuda")
        done = torch.zeros(1, dtype=torch.int32, device="cuda")
        plan.round_trips(Ap, As, None, pump, 0, 0, max_rt, ps_hist=hist, tol=tol, rt_done=done)
        torch.cuda.synchronize()
        n = int(done.item())
        return n, float(hist[n - 1].item()), p, (w, T)


def test_gpu_dro_steady_state_scales_as_sqrt_pump_ratio():
    n_ref, ps_ref, _, _ = gpu_steady(2.25)
    assert n_ref < 20000
    for n_thr, ratio in ((1.5625, 0.5), (4.0, 2.0), (6.25, 3.0)):
        n, ps, _, _ = gpu_steady(n_thr)
        assert n < 20000
        assert abs(ps / ps_ref / ratio - 1.0) < 0.05, (n_thr, ps / ps_ref)


def test_gpu_steady_state_matches_fp64_oracle():
    """Same start: the FP32 GPU steady state (relative power change per round
    trip below 1e-7, the FP32 resolution) is the FP64 one (converged to
    1e-10) within 1e-4."""
    n, ps, p, (w, T) = gpu_steady(4.0)
    As = np.full(p.n_t, 1e-2 + 0j)
    Ap = np.zeros(p.n_t, np.complex128)
    pump = np.full(p.n_t, np.float32(p.ap0), np.complex128)
    rts, ps64, conv = ob.solve(p, w.astype(np.float64), T.astype(np.float64), Ap, As, None, pump, 0, 20000, 1e-10)
    assert conv
    assert abs(ps - ps64) / ps64 < 1e-4, (ps, ps64, n, rts)
