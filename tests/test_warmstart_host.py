"""Host-side pieces of the learned warm start (no GPU): the band-centre code,
the flat parameter layout (biases) against the FP64 oracle's, and the
feature normalisation of the sweep's ranges."""
import numpy as np

from cuopo_b200 import sweep
from cuopo_b200 import warmstart as ws
from oracle import mlp_oracle as mo


def test_band_centre_code_round_trips_every_centre():
    n_t = 8192
    q0 = np.arange(ws.BAND // 2, n_t // 2 - ws.BAND // 2 + 1)
    code = ws.centre_code(q0.astype(np.float64), n_t).astype(np.float32)
    assert np.all(np.abs(code) <= 1.0)
    assert np.array_equal(ws.centre_decode(code, n_t), q0)


def test_bias_mask_matches_the_oracle_layout():
    for n_in, width, depth, n_out in [(4, 512, 4, 512), (3, 256, 2, 384)]:
        dims = mo.layer_dims(n_in, width, depth, n_out)
        mask = ws._bias_mask(n_in, width, depth, n_out)
        assert mask.size == mo.param_count(dims)
        p = np.arange(mask.size, dtype=np.float64)
        biases = np.concatenate([b for _, b in mo.unpack(p, dims)])
        assert np.array_equal(p[mask], biases)


def test_features_span_the_sweep_ranges():
    _, _, table = sweep.random_cw_sweep(256, 3, n_t_choices=(8192,))
    f = ws.features(table)
    assert f.shape == (256, ws.N_FEATURES) and f.dtype == np.float32
    assert np.all(np.abs(f) <= 1.0 + 1e-6)
    assert np.all(f.max(axis=0) > 0.8) and np.all(f.min(axis=0) < -0.8)
