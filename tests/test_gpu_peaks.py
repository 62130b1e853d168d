"""hj_measure_peaks: the library's own pipe-peak kernels run and give plausible
B200 figures (the roofline denominators the benchmark reports)."""
import pytest

pytestmark = pytest.mark.gpu


def test_measured_peaks_are_plausible(cuda):
    import hegjoin_b200 as hj
    p = hj.measure_peaks()
    assert 20 < p["fp32_fma_tflops"] < 400
    assert p["fp32_fma_tflops"] * 0.8 < p["fp32x2_fma_tflops"] < 800
    assert 1 < p["fp64_fma_tflops"] < 200
    for k in ("f16_mma_tflops", "bf16_mma_tflops"):
        assert 300 < p[k] < 5000, (k, p[k])
