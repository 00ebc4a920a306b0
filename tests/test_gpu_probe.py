"""The roofline denominators: measured FP32 and FP64 FMA throughput."""
import math

import pytest

import cuopo_b200 as cu

pytestmark = pytest.mark.gpu


def test_fma_probes():
    f32 = cu.probe_fp32_peak()
    f64 = cu.probe_fp64_peak()
    assert math.isfinite(f32) and math.isfinite(f64)
    # a B200 at any clock the driver allows: tens of FP32 TFLOP/s
    assert 10.0 < f32 < 200.0
    # the FP64 pipe is slower than the FP32 one (packed FP32x2 included)
    assert 0.01 * f32 < f64 < f32
