"""The kernel autotuner (cuopo_autotune): it picks among the built kernel
configurations of a grid size by timing them, and the choice changes only
the launch shape, not the results beyond FP32 rounding."""
import numpy as np
import pytest

import cuopo_b200 as cu
from cuopo_b200 import sweep

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

# (points per CTA, CTAs per cluster) built for 2-eq FP32 grids with a choice
CANDIDATES = {8192: {(4096, 2), (8192, 1)}, 16384: {(4096, 4), (8192, 2)}, 32768: {(4096, 8), (8192, 4)}}


def base_for(n_t):
    p, _ = cu.derive_params(sweep.cw_base_inputs(n_t=n_t, n_z=20, n_thr=3.0, r_percent=95.0))
    return p


def run_batch(n_t, count=8, n_rt=3):
    base = base_for(n_t)
    insts = [dict(n_t=n_t, ap0=base.ap0 * (1 + 0.1 * k), Rs=0.95, delta=0.01 * k, gdd=1e-5 * k, seed=k)
             for k in range(count)]
    with cu.Batch(base, insts) as b:
        init = torch.from_numpy(np.concatenate(
            [0.3 * np.exp(2j * np.pi * np.random.default_rng(k).random(n_t)) for k in range(count)])
            .astype(np.complex64)).cuda()
        b.set_signal(init)
        b.run(n_rt, 0.0)
        out = torch.empty_like(init)
        b.get_signal(out)
        ps, rts, flags = b.results()
    return out.cpu().numpy(), ps, rts


@pytest.fixture(autouse=True)
def _reset():
    cu.autotune_reset()
    yield
    cu.autotune_reset()


def test_single_candidate_needs_no_timing():
    r = cu.autotune(base_for(4096), cu.F32, count=4, n_rt=1)
    assert (r["points_per_cta"], r["cluster"]) == (4096, 1) and r["ms"] == -1.0


@pytest.mark.parametrize("n_t", sorted(CANDIDATES))
def test_choice_is_a_candidate_and_sticks(n_t):
    default = cu.kernel_config(n_t)
    assert default in CANDIDATES[n_t]
    r = cu.autotune(base_for(n_t), cu.F32, count=16, n_rt=1)
    choice = (r["points_per_cta"], r["cluster"])
    assert choice in CANDIDATES[n_t] and r["ms"] > 0
    assert cu.kernel_config(n_t) == choice
    cu.autotune_reset()
    assert cu.kernel_config(n_t) == default


def test_results_do_not_depend_on_the_choice():
    """The same batch on both 2^15 configurations: the fields agree to FP32
    rounding (5e-6 relative L2 after 3 round trips), the round trips match."""
    n_t = 32768
    outs = []
    for m, cl in sorted(CANDIDATES[n_t]):
        cu.kernel_select(n_t, m, cl)
        assert cu.kernel_config(n_t) == (m, cl)
        outs.append(run_batch(n_t))
    a, b = outs
    assert np.linalg.norm(a[0] - b[0]) / np.linalg.norm(b[0]) < 5e-6
    assert np.array_equal(a[2], b[2])
    assert np.max(np.abs(a[1] - b[1]) / b[1]) < 1e-5


def test_select_rejects_configurations_not_built():
    with pytest.raises(cu.CuopoError) as e:
        cu.kernel_select(32768, 2048, 16)
    assert e.value.status == cu.EUNSUPPORTED


def test_unsupported_grid_is_rejected():
    p = base_for(4096)
    p.n_t = 3000
    with pytest.raises(cu.CuopoError) as e:
        cu.autotune(p, cu.F32, count=4, n_rt=1)
    assert e.value.status == cu.EUNSUPPORTED
