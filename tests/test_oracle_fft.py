"""Pins the oracle's transforms to the FFTW conventions the reference relies on,
using scipy.fft (pocketfft) as the independent implementation:
- unnormalised complex DFT, sign -1 forward / +1 backward (fftwwrapper.hh plans);
- R2C with the halved dimension being parafields dimension 0 (r2cfieldbackend.hh:220-231);
- C2R ignoring Im at DC/Nyquist, complex transforms over the other dims first
  (r2cfieldbackend.hh:250-274 on non-Hermitian noise planes);
- REDFT00 == DCT-I (dctmatrixbackend.hh:252-266).
"""
import numpy as np
import pytest
import scipy.fft as sf


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 8, 12, 30, 49, 97, 121, 210, 1000, 1024, 2039, 4078])
def test_complex_fft(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(oracle.fft(x, -1), sf.fft(x), rtol=0, atol=1e-12 * max(1, np.abs(x).sum()))
    np.testing.assert_allclose(oracle.fft(x, +1), sf.ifft(x) * n, rtol=0, atol=1e-12 * max(1, np.abs(x).sum()))


@pytest.mark.parametrize("shape", [(16,), (6, 8), (10, 12, 8), (5, 7, 9), (4, 6, 10), (3, 22)])
def test_r2c_c2r_dct(oracle, shape):
    rng = np.random.default_rng(sum(shape))
    x = rng.standard_normal(shape)
    X = oracle.r2c(x)
    np.testing.assert_allclose(X, sf.rfftn(x), atol=1e-11)
    # non-Hermitian input: FFTW/pocketfft c2r semantics
    Xn = rng.standard_normal(X.shape) + 1j * rng.standard_normal(X.shape)
    np.testing.assert_allclose(oracle.c2r(Xn, shape[-1]), sf.irfftn(Xn, s=shape) * np.prod(shape), atol=1e-10)
    d = rng.standard_normal(tuple(s // 2 + 1 for s in shape))
    np.testing.assert_allclose(oracle.dct1(d), sf.dctn(d, type=1), atol=1e-11)


def test_fft_axis(oracle):
    rng = np.random.default_rng(3)
    x = rng.standard_normal((5, 6, 7)) + 1j * rng.standard_normal((5, 6, 7))
    for ax_param, ax_np in [(0, 2), (1, 1), (2, 0)]:
        np.testing.assert_allclose(oracle.fft_axis(x, ax_param, -1), sf.fft(x, axis=ax_np), atol=1e-12)
