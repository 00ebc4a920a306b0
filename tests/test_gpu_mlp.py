"""The warm-start network on the tensor cores (cuopo_gemm_bf16, cuopo_mlp_*)
against the FP64 CPU oracle (oracle/mlp_oracle.py), through the C ABI.

Tolerances (relative L2 unless stated):
* GEMM (BF16 operands, FP32 accumulation) vs FP64 of the same BF16 values: 2e-5;
* forward output vs the oracle emulating the GPU's BF16 storage: 2e-3, vs the
  pure FP64 network: 3e-2 (BF16 rounding of weights and activations);
* loss: 1e-3 relative; gradients per tensor vs the emulating oracle: 2e-2;
* an Adam step on the GPU's own gradient vs the oracle's Adam: 1e-5 of lr
  per parameter (FP32 arithmetic), except for gradients within FP32 noise of zero.
"""
import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _bf16_tensor(a):
    return torch.from_numpy(np.asarray(a, np.float32)).cuda().to(torch.bfloat16)


def _rel(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("M,N,K,split", [(128, 64, 64, 1), (256, 128, 512, 1), (4096, 512, 512, 1),
                                         (512, 64, 4096, 32), (512, 512, 4096, 8), (384, 192, 320, 5)])
def test_gemm_matches_fp64(M, N, K, split):
    from cuopo_b200 import warmstart as ws
    rng = np.random.default_rng(M + N + K)
    A = mo.bf16(rng.standard_normal((M, K)))
    B = mo.bf16(rng.standard_normal((N, K)))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    C = ws.gemm_bf16(_bf16_tensor(A), _bf16_tensor(B), split=split, err=err)
    torch.cuda.synchronize()
    assert err.item() == 0
    assert _rel(C.cpu().numpy(), A @ B.T) < 2e-5


def test_gemm_bounded_wait_reports_timeout_and_context_survives():
    """The test hook leaves each tile's completion barrier unsignalled: the
    epilogue's bounded wait (about 1 s) runs out, the error word gets bit 0,
    the output is not written, and the next GEMM on the same context is right."""
    from cuopo_b200 import warmstart as ws
    rng = np.random.default_rng(1)
    A = mo.bf16(rng.standard_normal((128, 64)))
    B = mo.bf16(rng.standard_normal((64, 64)))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.full((128, 64), 7.0, dtype=torch.float32, device="cuda")
    ws.gemm_bf16(_bf16_tensor(A), _bf16_tensor(B), err=err, flags=1, out=out)
    torch.cuda.synchronize()
    assert err.item() & 1
    assert torch.all(out == 7.0)
    err.zero_()
    C = ws.gemm_bf16(_bf16_tensor(A), _bf16_tensor(B), err=err)
    torch.cuda.synchronize()
    assert err.item() == 0 and _rel(C.cpu().numpy(), A @ B.T) < 2e-5


def _net(n_in, width, depth, n_out, batch, seed):
    from cuopo_b200 import warmstart as ws
    mlp = ws.MLP(n_in, width, depth, n_out, max_batch=batch, seed=seed)
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (batch, n_in)).astype(np.float32)
    t = (0.5 * rng.standard_normal((batch, n_out))).astype(np.float32)
    return mlp, x, t


SHAPES = [(4, 128, 2, 128, 256), (4, 512, 4, 512, 4096), (3, 256, 3, 384, 200)]


@pytest.mark.parametrize("n_in,width,depth,n_out,batch", SHAPES)
def test_forward_matches_oracle(n_in, width, depth, n_out, batch):
    mlp, x, _ = _net(n_in, width, depth, n_out, batch, 5)
    y = mlp.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    p = mlp.get_params().astype(np.float64)
    dims = mo.layer_dims(n_in, width, depth, n_out)
    y_emu, _ = mo.forward(p, x, dims, emulate_bf16=True)
    y_64, _ = mo.forward(p, x, dims, emulate_bf16=False)
    mlp.close()
    assert _rel(y, y_emu) < 2e-3
    assert _rel(y, y_64) < 3e-2


@pytest.mark.parametrize("n_in,width,depth,n_out,batch", SHAPES)
def test_gradients_match_oracle(n_in, width, depth, n_out, batch):
    mlp, x, t = _net(n_in, width, depth, n_out, batch, 7)
    loss, g = mlp.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    p = mlp.get_params().astype(np.float64)
    mlp.close()
    dims = mo.layer_dims(n_in, width, depth, n_out)
    loss_ref, g_ref = mo.loss_and_grads(p, x, t, dims, emulate_bf16=True)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    o = 0
    for l, (n, k) in enumerate(dims):
        gw, gw_ref = g[o:o + n * k], g_ref[o:o + n * k]
        o += n * k
        gb, gb_ref = g[o:o + n], g_ref[o:o + n]
        o += n
        assert _rel(gw, gw_ref) < 2e-2, (l, "W", _rel(gw, gw_ref))
        assert _rel(gb, gb_ref) < 2e-2, (l, "b", _rel(gb, gb_ref))


def test_adam_step_matches_oracle():
    mlp, x, t = _net(4, 128, 2, 128, 256, 11)
    X, T = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    _, g = mlp.gradients(X, T)
    p0 = mlp.get_params().astype(np.float64)
    lr = 1e-3
    mlp.train_step(X, T, lr)
    mlp.status()
    p1 = mlp.get_params().astype(np.float64)
    mlp.close()
    ref = mo.adam_step(p0.copy(), g.astype(np.float64), np.zeros_like(p0), np.zeros_like(p0), 1, lr)
    d = np.abs(p1 - ref)
    tiny = np.abs(g) < 1e-6 * np.max(np.abs(g))   # sign of a gradient within FP32 noise of zero
    assert np.all(d[~tiny] <= 1e-5 * lr + 1e-7 * np.abs(p0[~tiny]))
    assert np.mean(tiny) < 0.01


def test_training_fits_a_smooth_map():
    """Adam through the captured training graph fits y = sin/cos features of x."""
    from cuopo_b200 import warmstart as ws
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, (2048, 4)).astype(np.float32)
    freq = rng.standard_normal((4, 64))
    t = np.concatenate([np.sin(x @ freq), np.cos(x @ freq)], axis=1).astype(np.float32)
    mlp = ws.MLP(4, 256, 3, 128, max_batch=1024, seed=3)
    losses = ws.train(mlp, x, t, steps=400, batch=1024, lr=2e-3)
    mlp.close()
    assert np.all(np.isfinite(losses))
    assert losses[-20:].mean() < 0.1 * losses[:5].mean()


def _modes(seed):
    from cuopo_b200 import warmstart as ws
    rng = np.random.default_rng(seed)
    m = (rng.standard_normal((6, 2 * ws.N_MODES)) * np.exp(-np.abs(np.arange(2 * ws.N_MODES) - ws.N_MODES) / 40))
    m[:, ws.N_MODES] = 3.0          # dominant mode 0 (the 2k-th pair is mode k - 128), real part > 0
    return m.astype(np.float32)


@pytest.mark.parametrize("n_t", [512, 4096, 16384, 32768])
def test_fields_from_modes_matches_fp64_synthesis(n_t):
    """The direct synthesis kernel against numpy's FP64 sum of the modes."""
    from cuopo_b200 import warmstart as ws
    m = _modes(n_t)
    f = ws.modes_to_fields(torch.from_numpy(m).cuda(), n_t, scale=2.0).cpu().numpy()
    c = m[:, 0::2].astype(np.float64) + 1j * m[:, 1::2]
    q = np.arange(ws.N_MODES) - ws.N_MODES // 2
    n = np.arange(n_t)
    ref = 2.0 * c @ np.exp(2j * np.pi * np.outer(q, n) / n_t)
    assert _rel(f, ref) < 5e-6


@pytest.mark.parametrize("n_t", [4096, 8192])
def test_modes_fields_round_trip(n_t):
    """modes -> field (direct synthesis) -> modes (own FFT) returns the
    modes; a field and its negative give the same canonical modes."""
    from cuopo_b200 import warmstart as ws
    m = _modes(n_t)
    f = ws.modes_to_fields(torch.from_numpy(m).cuda(), n_t, scale=2.0)
    back = ws.fields_to_modes(f, n_t, scale=2.0)
    back_neg = ws.fields_to_modes(-f, n_t, scale=2.0)
    torch.cuda.synchronize()
    assert _rel(back.cpu().numpy(), m) < 1e-5
    assert _rel(back_neg.cpu().numpy(), m) < 1e-5
    # the field itself: its mean is mode 0 times the scale
    assert abs(f.mean(dim=1)[0].item() - 2.0 * complex(m[0, 256], m[0, 257])) < 1e-4


def test_band_targets_and_synthesis_round_trip():
    """A field made of two bands around +-q0 whose pairs c_q c_-q share the
    phase Phi: band_targets recovers q0, Phi and the power, and
    cuopo_fields_from_bands rebuilds a field with the same band power
    spectrum, power and pair phase (FFT of the library)."""
    from cuopo_b200 import api
    from cuopo_b200 import warmstart as ws
    n_t, q0, phi, P = 8192, 2500, 0.9, 0.6
    rng = np.random.default_rng(4)
    k = np.arange(ws.BAND) - ws.BAND // 2
    mag = np.exp(-(k / 20.0) ** 2)
    spec = np.zeros(n_t, np.complex128)
    psi = rng.uniform(-np.pi, np.pi, ws.BAND)          # in-band relative phases (not predicted)
    spec[(q0 + k) % n_t] = mag * np.exp(1j * (phi / 2 + psi))
    spec[(-q0 - k) % n_t] = mag * np.exp(1j * (phi / 2 - psi))
    spec *= np.sqrt(P / np.sum(np.abs(spec) ** 2))
    field = np.fft.ifft(spec) * n_t                    # A[n] = sum_q c_q e^{+2 pi i q n / N}
    F = torch.from_numpy(field.astype(np.complex64)).cuda()[None, :]
    y, q_found = ws.band_targets(F, np.array([P]), n_t)
    assert int(q_found[0]) == q0
    yy = y.cpu().numpy()[0]
    assert abs(np.arctan2(yy[320:384].mean(), yy[256:320].mean()) - phi) < 1e-4
    assert abs(10 ** yy[448:512].mean() - P) < 1e-5 * P
    out = torch.empty(1, n_t, dtype=torch.complex64, device="cuda")
    from cuopo_b200._lib import check, load
    check(load().cuopo_fields_from_bands(y.data_ptr(), 1, n_t, 1.0, out.data_ptr(), None,
                                         torch.cuda.current_stream().cuda_stream))
    c = api.fft_c2c(out.contiguous(), -1).cpu().numpy()[0] / n_t
    assert abs(np.sum(np.abs(c) ** 2) - P) < 1e-4 * P
    got = np.abs(c[(q0 + k) % n_t])
    want = np.abs(spec[(q0 + k) % n_t])
    assert _rel(got, want) < 1e-4
    pairs = c[(q0 + k) % n_t] * c[(-q0 - k) % n_t]
    assert abs(np.angle(pairs.sum()) - phi) < 1e-4


def test_grad_step_and_adam_equal_train_step():
    """The data-parallel pieces (cuopo_mlp_grad_step, the gradient buffer,
    cuopo_mlp_apply_adam) take the same steps as cuopo_mlp_train_step on
    one rank; the gradient buffer is the device view the all-reduce uses."""
    from cuopo_b200 import warmstart as ws
    rng = np.random.default_rng(12)
    x = torch.from_numpy(rng.uniform(-1, 1, (256, 4)).astype(np.float32)).cuda()
    t = torch.from_numpy((0.5 * rng.standard_normal((256, 128))).astype(np.float32)).cuda()
    a = ws.MLP(4, 128, 2, 128, max_batch=256, seed=21)
    b = ws.MLP(4, 128, 2, 128, max_batch=256, seed=21)
    lr = 1e-3
    for _ in range(3):
        a.train_step(x, t, lr)
        b.grad_step(x, t)
        g = b.grad_tensor()
        assert g.is_cuda and g.numel() >= b.n_params
        g.mul_(2.0)                      # as after a sum over two identical ranks ...
        b.apply_adam(lr, grad_scale=0.5)  # ... and the mean
    a.status()
    b.status()
    pa, pb = a.get_params(), b.get_params()
    a.close()
    b.close()
    assert np.max(np.abs(pa - pb)) <= 1e-5 * lr * 3 + 1e-6 * np.max(np.abs(pa))
