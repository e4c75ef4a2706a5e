"""Edge cases through the C ABI on the GPU: degenerate and ragged grids against the oracle,
configuration errors with the reference's messages, the extended-domain size limit, empty
batches and null arguments."""
import ctypes as C

import numpy as np
import pytest

import pfb200
from helpers import desc_of, rel

pytestmark = pytest.mark.gpu

EDGE = {
    # one cell along an axis: a torus of 2 along it (transforms of length 2 and 1)
    "2d-one-row": dict(dim=2, cells=(64, 1), covariance="exponential", corr_length=0.1),
    "2d-one-col": dict(dim=2, cells=(1, 48), covariance="gaussian", corr_length=0.3, approximate=True),
    "3d-one-plane": dict(dim=3, cells=(12, 10, 1), covariance="matern32", corr_length=0.2, approximate=True),
    # smallest 3D grid, ragged odd sizes (pencil tiles and pairs with a missing partner)
    "3d-2cubed": dict(dim=3, cells=(2, 2, 2), covariance="exponential", corr_length=0.5),
    "3d-ragged-odd": dict(dim=3, cells=(33, 17, 9), covariance="spherical", corr_length=0.3, approximate=True),
    "2d-ragged-prime": dict(dim=2, cells=(7, 11), covariance="exponential", corr_length=(0.2, 0.1),
                            anisotropy="axiparallel"),
    # factor 3 on even cells: even torus, R2C with a pitch that is not a power of two
    "2d-factor3": dict(dim=2, cells=(20, 14), covariance="exponential", corr_length=0.2, embedding_factor=3),
    # periodic: embedding factor 1
    "2d-periodic": dict(dim=2, cells=(32, 24), covariance="exponential", corr_length=0.05, periodic=True,
                        approximate=True),
}


@pytest.mark.parametrize("prec", [pfb200.PREC_F64, pfb200.PREC_F32])
@pytest.mark.parametrize("name", list(EDGE))
def test_degenerate_and_ragged_grids(oracle, name, prec):
    d = desc_of(EDGE[name], precision=prec)
    lam, st, status = oracle.spectrum(d)
    assert status == 0
    P = pfb200.Plan(d)
    gst = P.spectrum_build()
    assert (gst["small"], gst["zero"], gst["negative"]) == (st["small"], st["zero"], st["negative"])
    assert rel(P.spectrum(), lam) < 1e-12
    g = oracle.resolve(d)
    noise = oracle.noise(2, g.noise)
    ref, _ = oracle.generate(d, lam, noise)
    tol = 1e-11 if prec == pfb200.PREC_F64 else 1e-5
    assert rel(P.generate(noise=noise), ref) < tol
    x = np.random.default_rng(1).standard_normal(g.domain)
    dt = np.float64 if prec == pfb200.PREC_F64 else np.float32
    out = P.matvec(x.astype(dt), op=pfb200.OP_MUL, precision=prec)
    assert rel(out, oracle.matvec(d, lam, pfb200.OP_MUL, x)) < (1e-12 if prec == pfb200.PREC_F64 else 1e-5)
    P.close()


@pytest.mark.parametrize("over,msg", [
    (dict(dim=2, cells=(15, 8), embedding_factor=3), "even number of extended cells"),
    (dict(dim=3, cells=(8, 8, 8), covariance="cubic"), "cubic covariance only applicable"),
    (dict(dim=2, cells=(8, 8), covariance="gammaExponential", exp_gamma=2.5), "between 0 and 2"),
    (dict(dim=2, cells=(8, 8), covariance="generalizedCauchy", cauchy_alpha=2.5, cauchy_beta=1.0),
     "alpha has to be in range"),
    (dict(dim=2, cells=(8, 8), covariance="matern", matern_nu=-1.0), "matern nu has to be positive"),
    (dict(dim=2, cells=(0, 8)), "grid.cells must be positive"),
    (dict(dim=1, cells=(16,), matrix_backend=pfb200.MATRIX_DCT), "dim 1 requires"),
    (dict(dim=2, cells=(8, 8), matrix_backend=pfb200.MATRIX_R2C, field_backend=pfb200.FIELD_DFT),
     "cannot serve DFTFieldBackend"),
    (dict(dim=2, cells=(8, 8), matrix_backend=pfb200.MATRIX_R2C, field_backend=pfb200.FIELD_DCTDST),
     "requires DCTMatrixBackend"),
])
def test_configuration_errors(over, msg):
    cfg = dict(covariance="exponential", corr_length=0.1)
    cfg.update(over)
    with pytest.raises(pfb200.PfError, match=msg) as e:
        pfb200.Plan(desc_of(cfg))
    assert e.value.status == pfb200.PF_ERR_CONFIG


def test_extended_domain_limit():
    """fieldtraits.hh keeps cell indices in 32-bit unsigned integers: a torus of more than 2^32
    cells is refused before anything is allocated."""
    with pytest.raises(pfb200.PfError, match="2\\^32") as e:
        pfb200.Plan(desc_of(dict(dim=3, cells=(1024, 1024, 1024), covariance="exponential", corr_length=0.1)))
    assert e.value.status == pfb200.PF_ERR_CONFIG


def test_empty_batches_and_null_arguments():
    torch = pytest.importorskip("torch")
    L = pfb200.lib()
    P = pfb200.Plan(desc_of(dict(dim=2, cells=(16, 16), covariance="exponential", corr_length=0.1)))
    buf = torch.empty(16 * 16, dtype=torch.float64, device="cuda")
    assert L.pf_generate_batch(P.h, 1, 0, buf.data_ptr(), pfb200.MEM_DEVICE, 0) == pfb200.PF_OK
    assert L.pf_multiply_inverse_batch(P.h, None, None, 0, pfb200.MEM_DEVICE, None, None, 2) == pfb200.PF_OK
    assert L.pf_matvec(P.h, 0, 0, None, buf.data_ptr(), pfb200.MEM_DEVICE) == pfb200.PF_ERR_ARG
    assert L.pf_generate_batch(P.h, 1, -1, buf.data_ptr(), pfb200.MEM_DEVICE, 0) == pfb200.PF_ERR_ARG
    assert L.pf_spectrum_build_values(P.h, None, 0, pfb200.MEM_HOST, None) == pfb200.PF_ERR_ARG
    st = pfb200.EigStats()
    assert L.pf_spectrum_build(None, C.byref(st)) == pfb200.PF_ERR_ARG
    with pytest.raises(ValueError, match="buffer"):
        P.generate(out=torch.empty(10, dtype=torch.float64, device="cuda"))
    P.close()
