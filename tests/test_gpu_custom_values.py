"""pf_spectrum_build_values: fillTransformedMatrix with covariance values the caller
computed (the custom-iso / custom-aniso covariances, matrix.hh:223-265,
randomfield.hh:430-451).  Values of the built-in covariances filled by the oracle in each
matrix backend's layout give the oracle's spectrum and realizations; a custom plan
without values, and values of the wrong count, are refused."""
import numpy as np
import pytest

import pfb200
from helpers import desc_of, rel

pytestmark = pytest.mark.gpu

CASES = {
    "2d-dct-exp": dict(dim=2, cells=(64, 48), covariance="exponential", corr_length=0.1),
    "3d-dct-m32-axi": dict(dim=3, cells=(32, 24, 20), covariance="matern32", corr_length=(0.2, 0.1, 0.05),
                           anisotropy="axiparallel", approximate=True),
    "2d-r2c-sph-geo": dict(dim=2, cells=(50, 36), covariance="spherical", corr_length=(0.2, 0.05, -0.05, 0.15),
                           anisotropy="geometric", approximate=True),
    "3d-r2c-exp-geo": dict(dim=3, cells=(24, 20, 16), covariance="exponential",
                           corr_length=(0.15, 0.02, 0.0, -0.03, 0.08, 0.01, 0.0, 0.02, 0.04),
                           anisotropy="geometric", approximate=True),
    "2d-dft-m52": dict(dim=2, cells=(24, 20), covariance="matern52", corr_length=0.15,
                       matrix_backend=pfb200.MATRIX_DFT, field_backend=pfb200.FIELD_DFT),
}


def matrix_values(oracle, d):
    """the matrix cells of the built-in covariance, dense, dimension 0 fastest"""
    g = oracle.resolve(d)
    v = oracle.fill_matrix(d)
    if g.matrix_backend == pfb200.MATRIX_R2C:  # drop the two padding entries per row
        T0 = g.T[0]
        v = v.reshape(-1, 2 * (T0 // 2 + 1))[:, :T0].ravel()
    return np.ascontiguousarray(v)


@pytest.mark.parametrize("prec", [pfb200.PREC_F64, pfb200.PREC_F32])
@pytest.mark.parametrize("name", list(CASES))
def test_values_give_the_builtin_spectrum_and_field(oracle, name, prec):
    cfg = CASES[name]
    d = desc_of(cfg, precision=prec)
    lam, st, _ = oracle.spectrum(d)
    P = pfb200.Plan(desc_of(cfg, precision=prec, covariance="custom-iso"))
    gst = P.spectrum_build_values(matrix_values(oracle, d))
    assert (gst["small"], gst["zero"], gst["negative"]) == (st["small"], st["zero"], st["negative"])
    assert rel(P.spectrum(), lam) < 1e-12
    g = oracle.resolve(d)
    noise = oracle.noise(31, g.noise)
    ref, _ = oracle.generate(d, lam, noise)
    assert rel(P.generate(noise=noise), ref) < (1e-11 if prec == pfb200.PREC_F64 else 1e-5)
    P.close()


def test_values_from_device_memory(oracle):
    torch = pytest.importorskip("torch")
    cfg = CASES["3d-r2c-exp-geo"]
    d = desc_of(cfg)
    lam, _, _ = oracle.spectrum(d)
    P = pfb200.Plan(desc_of(cfg, covariance="custom-aniso"))
    P.spectrum_build_values(torch.from_numpy(matrix_values(oracle, d)).cuda())
    assert rel(P.spectrum(), lam) < 1e-12
    P.close()


def test_custom_plan_needs_values(oracle):
    cfg = CASES["2d-dct-exp"]
    P = pfb200.Plan(desc_of(cfg, covariance="custom-iso"))
    with pytest.raises(pfb200.PfError, match="fillMatrix"):
        P.spectrum_build()
    with pytest.raises(pfb200.PfError, match="covariance values"):
        P.spectrum_build_values(np.ones(10))
    with pytest.raises(pfb200.PfError, match="fillMatrix"):
        P.generate(seed=1)
    P.close()


def test_custom_negative_eigenvalues_raise(oracle):
    """the NegativeEigenvalueError rule applies to caller values as to built-in ones"""
    cfg = dict(dim=2, cells=(32, 32), covariance="gaussian", corr_length=0.5)
    d = desc_of(cfg)
    P = pfb200.Plan(desc_of(cfg, covariance="custom-iso"))
    with pytest.raises(pfb200.NegativeEigenvalueError):
        P.spectrum_build_values(matrix_values(oracle, d))
    P.close()
