"""GPU FFT (cuopo_fft_c2c, the cufftExecC2C stand-in) against numpy in FP64 and
against cuFFT (torch.fft) on the same inputs.

Bars: F64 transforms within 1e-13 relative L2 of numpy; F32 transforms within
1.5x cuFFT's own error (and below 3e-7) relative to numpy's FP64 result."""
import numpy as np
import pytest

import cuopo_b200 as cu
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def batch(n, b, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((b, n)) + 1j * rng.standard_normal((b, n))


@pytest.mark.parametrize("n", [512, 1024, 2048, 4096, 8192])
@pytest.mark.parametrize("sign", [1, -1])
def test_fft_f32_vs_numpy_and_cufft(n, sign):
    x = batch(n, 64, n + sign)
    xd = torch.from_numpy(x.astype(np.complex64)).cuda()
    got = cu.fft_c2c(xd, sign).cpu().numpy()
    x32 = x.astype(np.complex64).astype(np.complex128)
    ref = np.fft.ifft(x32, axis=-1) * n if sign > 0 else np.fft.fft(x32, axis=-1)
    cufft = (torch.fft.ifft(xd, dim=-1, norm="forward") if sign > 0 else torch.fft.fft(xd, dim=-1)).cpu().numpy()
    e_ours = rel_l2(got, ref)
    e_cufft = rel_l2(cufft, ref)
    assert e_ours < max(1.5 * e_cufft, 1e-7) and e_ours < 3e-7, (e_ours, e_cufft)


@pytest.mark.parametrize("n", [512, 1024, 2048, 4096])
def test_fft_f64_vs_numpy(n):
    x = batch(n, 8, n)
    xd = torch.from_numpy(x).cuda()
    for sign in (1, -1):
        got = cu.fft_c2c(xd, sign).cpu().numpy()
        ref = np.fft.ifft(x, axis=-1) * n if sign > 0 else np.fft.fft(x, axis=-1)
        assert rel_l2(got, ref) < 1e-13


def test_fft_in_place_and_round_trip():
    n = 4096
    x = batch(n, 5, 1)
    xd = torch.from_numpy(x).cuda()
    y = xd.clone()
    cu.fft_c2c(y, -1, out=y)
    cu.fft_c2c(y, +1, out=y)
    assert rel_l2(y.cpu().numpy() / n, x) < 1e-14


def test_fft_rejects_bad_sizes():
    x = torch.zeros(3 * 512, dtype=torch.complex64, device="cuda").reshape(3, 512)
    with pytest.raises(cu.CuopoError):
        cu.fft_c2c(torch.zeros(1000, dtype=torch.complex64, device="cuda"), 1)
    cu.fft_c2c(x, 1)
