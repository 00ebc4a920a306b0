"""The warm-start network's FP64 oracle (oracle/mlp_oracle.py) on the CPU:
its gradients against central finite differences of its own loss, and
the BF16 rounding helper against exact cases."""
import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding_exact_cases():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0, 3.0e-39], np.float64)
    got = mo.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1); 1 + 3 2^-8 rounds up to 1 + 2^-6
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1.0 + 2 ** -6 and got[3] == 1.0
    assert got[4] == -2.5 and got[5] == 0.0


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    dims = mo.layer_dims(4, 12, 3, 10)
    P = mo.param_count(dims)
    params = rng.standard_normal(P) * 0.4
    x = rng.standard_normal((7, 4))
    t = rng.standard_normal((7, 10))
    _, g = mo.loss_and_grads(params, x, t, dims, emulate_bf16=False)
    idx = rng.choice(P, 60, replace=False)
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        l1, _ = mo.loss_and_grads(p1, x, t, dims, emulate_bf16=False)
        l2, _ = mo.loss_and_grads(p2, x, t, dims, emulate_bf16=False)
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(fd), (i, fd, g[i])


def test_adam_first_step_moves_every_parameter_by_lr():
    p = np.array([1.0, -2.0, 0.5])
    g = np.array([0.3, -1e-3, 2.0])
    m = np.zeros(3)
    v = np.zeros(3)
    mo.adam_step(p, g, m, v, 1, 1e-2)
    # first bias-corrected step: m_hat / sqrt(v_hat) = sign(g)
    assert np.allclose(p, [1.0 - 1e-2, -2.0 + 1e-2, 0.5 - 1e-2], atol=1e-9)
