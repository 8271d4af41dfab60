"""h3c_fma_rates: the FP64 and FP32 fused multiply-add rates of the device,
measured with register-only FMA chains (the denominator for arithmetic-bound
stage kernels)."""
import pytest

pytestmark = pytest.mark.gpu


def test_fma_rates_are_plausible():
    from hom3_b200.solver import fma_rates
    r64, r32 = fma_rates()
    assert 1e12 < r64 < 1e15 and 1e12 < r32 < 1e15
    assert r32 > r64  # FP32 issues at least as fast as FP64 on every current data-centre GPU
    again = fma_rates()
    assert abs(again[0] - r64) <= 0.2 * r64
