"""The measured compute peaks used as roofline denominators are positive and ordered as the
hardware is (tensor TF32 > FP32 FMA > FP64 FMA on a B200)."""
import pytest

from gems_b200 import measure_peaks

pytestmark = pytest.mark.gpu


def test_measured_peaks(gpu):
    p = measure_peaks(0)
    assert 0 < p["fp64_tflops"] < p["fp32_tflops"] < p["tf32_tflops"]
    # orders of magnitude of a B200 (dense): tens of TFLOP/s on the CUDA cores, ~1 PFLOP/s TF32
    assert 5 < p["fp64_tflops"] < 200
    assert 20 < p["fp32_tflops"] < 400
    assert 200 < p["tf32_tflops"] < 5000
