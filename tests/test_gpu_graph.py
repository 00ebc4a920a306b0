"""Round trips captured in a CUDA graph: cuopo_round_trips issues only a
kernel launch on the caller's stream (no allocation, copy or
synchronisation), so a block of round trips can be captured once and
replayed.  Replays equal direct calls bit for bit."""
import numpy as np
import pytest

import cuopo_b200 as cu
from tests.helpers import params_2eq, params_3eq, random_field

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("neq,n_t", [(2, 2048), (2, 16384), (3, 1024)])
def test_graph_replays_equal_direct_calls(neq, n_t):
    p = params_2eq(n_t=n_t, n_z=6, gdd_percent=30.0) if neq == 2 else params_3eq(n_t=n_t, n_z=6, regime=cu.CW)
    T, w = cu.make_grids(p.n_t, p.t_rt)
    init = [random_field(n_t, 0.08, 1), random_field(n_t, 0.3, 2)] + ([random_field(n_t, 0.3, 3)] if neq == 3 else [])
    pump = torch.full((n_t,), complex(np.float32(p.ap0)), dtype=torch.complex64, device="cuda")
    dev = lambda: [torch.from_numpy(x.astype(np.complex64)).cuda() for x in init]
    n_blocks, per_block = 3, 2
    with cu.Plan(p, w, T, precision=cu.F32) as plan:
        # direct calls, each continuing from the fields the previous one left
        a = dev()
        hist_a = []
        for _ in range(n_blocks):
            h = torch.zeros(per_block, dtype=torch.float64, device="cuda")
            plan.round_trips(a[0], a[1], a[2] if neq == 3 else None, pump, 0, 0, per_block, ps_hist=h)
            hist_a.append(h.clone())
        torch.cuda.synchronize()
        # the same block captured once, replayed n_blocks times
        b = dev()
        h = torch.zeros(per_block, dtype=torch.float64, device="cuda")
        s = torch.cuda.Stream()
        warm = dev()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):      # first launch of this kernel outside the capture
            plan.round_trips(warm[0], warm[1], warm[2] if neq == 3 else None, pump, 0, 0, 1, stream=s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            plan.round_trips(b[0], b[1], b[2] if neq == 3 else None, pump, 0, 0, per_block, ps_hist=h,
                             stream=torch.cuda.current_stream())
        hist_b = []
        for _ in range(n_blocks):
            g.replay()
            hist_b.append(h.clone())
        torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    for x, y in zip(hist_a, hist_b):
        assert torch.equal(x, y)
