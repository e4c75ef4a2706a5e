"""pf_matvec_static: the matrix-vector product for callers that cannot allocate device
memory when they need the product -- code running inside another framework's memory pool
(which may own all of the GPU's memory), or a solver that reserves its memory once at
start-up and cannot accept the device synchronization of a later cudaMalloc.  Its scratch
is a fixed array inside the library, so the call itself allocates nothing.

Checked through the C ABI against the allocating entry point pf_matvec on two calls in
a row, and against the FP64 oracle, with the FP64 matvec tolerance of the parity tests;
the free device memory does not change across the calls.  This file is collected last on
purpose."""
import numpy as np
import pytest

import pfb200
from helpers import desc_of, rel

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


@pytest.mark.parametrize("cfg", [
    dict(dim=2, cells=(96, 80), covariance="exponential", corr_length=0.1),
    dict(dim=2, cells=(64, 72), covariance="spherical", corr_length=(0.2, 0.05, -0.05, 0.15),
         anisotropy="geometric", approximate=True),
], ids=["iso-dct", "geometric-r2c"])
@pytest.mark.parametrize("op", [pfb200.OP_MUL, pfb200.OP_ROOT, pfb200.OP_INVEXT])
def test_static_matvec_matches_pf_matvec(cfg, op, oracle):
    torch = pytest.importorskip("torch")
    L = pfb200.lib()
    d = desc_of(cfg)
    P = pfb200.Plan(d)
    P.spectrum_build()
    lam = P.spectrum()
    if op == pfb200.OP_INVEXT and (lam <= 0).any():
        pytest.skip("clamped zero eigenvalues make the torus inverse infinite")
    n = P.info.domain_size
    gen = torch.Generator(device="cuda").manual_seed(1)
    xs = [torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) for _ in range(2)]
    outs = [torch.empty_like(xs[0]) for _ in range(2)]
    # one call first: it looks up the array's device address and loads the kernels
    assert L.pf_matvec_static(P.h, op, xs[0].data_ptr(), outs[0].data_ptr()) == pfb200.PF_OK, \
        L.pf_last_error_string().decode()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for x, y in zip(xs, outs):  # two calls in a row
        assert L.pf_matvec_static(P.h, op, x.data_ptr(), y.data_ptr()) == pfb200.PF_OK, \
            L.pf_last_error_string().decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0  # nothing was allocated
    olam, _, _ = oracle.spectrum(d)
    for x, y in zip(xs, outs):
        ref = P.matvec(x, op=op, out=torch.empty_like(x))
        torch.cuda.synchronize()
        assert rel(y.cpu().numpy(), ref.cpu().numpy()) < TOL64
        assert rel(y.cpu().numpy(), oracle.matvec(d, olam, op, x.cpu().numpy())) < TOL64


def test_static_matvec_rejects_what_it_cannot_serve():
    torch = pytest.importorskip("torch")
    L = pfb200.lib()
    x = torch.zeros(1024 * 1024, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    P = pfb200.Plan(desc_of(dict(dim=2, cells=(64, 64), covariance="exponential", corr_length=0.1)))
    assert L.pf_matvec_static(P.h, 0, x.data_ptr(), y.data_ptr()) == pfb200.PF_ERR_STATE
    big = pfb200.Plan(desc_of(dict(dim=2, cells=(1024, 1024), covariance="exponential", corr_length=0.1)))
    big.spectrum_build()
    assert L.pf_matvec_static(big.h, 0, x.data_ptr(), y.data_ptr()) == pfb200.PF_ERR_ARG
    assert "static scratch" in L.pf_last_error_string().decode()
    # a torus length with a prime factor above 13 (2 x 17): no Bluestein transform here
    prime = pfb200.Plan(desc_of(dict(dim=2, cells=(17, 16), covariance="exponential", corr_length=0.1)))
    prime.spectrum_build()
    assert L.pf_matvec_static(prime.h, 0, x.data_ptr(), y.data_ptr()) == pfb200.PF_ERR_CONFIG
    # host memory is refused before any kernel could touch it
    hx = np.zeros(64 * 64)
    hy = np.zeros(64 * 64)
    P.spectrum_build()
    assert L.pf_matvec_static(P.h, 0, hx.ctypes.data, hy.ctypes.data) == pfb200.PF_ERR_ARG
    assert "device" in L.pf_last_error_string().decode()
