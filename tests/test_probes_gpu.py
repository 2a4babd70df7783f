"""The measurement probes the benchmark divides by (L2 read bandwidth, FP32
FMA rate) return figures in the range a B200 can reach."""
import pytest

import rayengine_b200 as rb

pytestmark = pytest.mark.gpu


def test_fp32_fma_rate_is_plausible(cuda):
    tops = rb.measure_fp32_fma_tops(1 << 16)
    # 148 SMs x 128 lanes x at most ~2 GHz = 37.9e12 FMAs/s; far below means
    # the probe does not keep the pipes busy, above means it skipped work
    assert 20.0 < tops < 40.0, tops


def test_l2_read_rate_is_plausible(cuda):
    gbs = rb.measure_l2_read_gbs(32 << 20, 50)
    # well above HBM (a few TB/s) and below an aggregate L2 limit of tens of TB/s
    assert 8000.0 < gbs < 40000.0, gbs
