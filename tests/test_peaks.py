"""pf_measure_peaks: the CUDA-core FMA microbenchmark behind the compute fractions of the
benchmark line returns positive, ordered throughputs (FP64 below FP32)."""
import pytest

import pfb200


@pytest.mark.gpu
def test_measure_peaks_plausible():
    p = pfb200.measure_peaks(0)
    assert p["sms"] > 0 and p["sm_clock_mhz"] > 0
    assert p["fp32_ffma_tflops"] > 1.0 and p["fp32_ffma2_tflops"] > 1.0
    assert 0.0 < p["fp64_dfma_tflops"] < max(p["fp32_ffma_tflops"], p["fp32_ffma2_tflops"])
    # the FFMA count of the kernels: at most 2 flops x 128 lanes (x2 for FFMA2) per SM per clock
    bound = 2 * 2 * 128 * p["sms"] * p["sm_clock_mhz"] * 1e6 / 1e12
    assert p["fp32_ffma2_tflops"] <= 1.05 * bound
