"""Host-side pieces of bench.py (no GPU): the reference arm draws the same
sweep as the product's sweep generator without importing the product, and
its set-up runs on the reference's own host code."""
import ast
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_draws_the_products_sweep():
    import bench
    from cuopo_b200 import sweep
    _, insts, table = sweep.random_cw_sweep(64, 0)
    t = bench.draw_sweep_table(64, 0)
    for k in ("n_thr", "delta_rad", "gdd_fs2", "refl", "n_t"):
        assert np.array_equal(np.asarray(t[k]), np.asarray(table[k])), k


def test_reference_arm_imports_nothing_of_the_product():
    """run_reference and the helpers it calls name no cuopo_b200 module."""
    src = (ROOT / "bench.py").read_text()
    tree = ast.parse(src)
    fns = {n.name: n for n in tree.body if isinstance(n, ast.FunctionDef)}
    for name in ("run_reference", "draw_sweep_table", "load_rts_record", "rts_by_size_from"):
        for node in ast.walk(fns[name]):
            if isinstance(node, ast.Import):
                assert not any(a.name.startswith("cuopo_b200") for a in node.names), name
            elif isinstance(node, ast.ImportFrom):
                assert not (node.module or "").startswith("cuopo_b200"), name
            elif isinstance(node, ast.Name):
                assert node.id not in ("cu", "sweep", "shard"), (name, node.id)


def test_flop_accounting_constants():
    """The algorithmic work per round trip behind `roofline.achieved`: per
    point and slice 10 F log2 N (forward and inverse transform of each field,
    5 N log2 N each) + 328 (the 2-equation RK4 half steps) + 12 (linear
    step), 600 for the 2^13 single CW OPO; per round trip 8 per point for the
    cavity map and, with GDD, one more transform pair and phase per point."""
    import bench
    n = 8192
    assert 10 * 2 * 13 + 328 + 12 == 600
    assert bench.flops_per_instance_rt(n, 0.0) == bench.N_Z * n * 600 + 8 * n
    assert bench.flops_per_instance_rt(n, 1e-4) == bench.N_Z * n * 600 + 8 * n + n * (10 * 13 + 6)
