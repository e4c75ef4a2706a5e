"""GPU parity: libpfcuda.so (through the C ABI) against the FP64 oracle on identical
seeded noise.  Tolerances (relative L2 unless stated):
  FP64 spectrum / matvec:         1e-12   (different FFT factorisations, both FP64)
  FP64 field:                     1e-11   (sqrt of eigenvalues near 1e-18 amplifies their
                                           1e-17 absolute roundoff)
  FP32 field / matvec:            1e-5    (FP32 transforms of an FP64 spectrum)
  eigenvalue statistics:          exact counts, smallest to 1e-12 relative
"""
import numpy as np
import pytest

import pfb200
from helpers import counter_noise, desc_of, rel

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL64F = 1e-11
TOL32 = 1e-5

CONFIGS = {
    "2d-exp-iso": dict(dim=2, cells=(64, 48), covariance="exponential", corr_length=0.1),
    "2d-cubic-axi": dict(dim=2, cells=(40, 72), covariance="cubic", corr_length=(0.3, 0.2),
                         anisotropy="axiparallel", extensions=(1.0, 2.0)),
    "2d-sph-geo": dict(dim=2, cells=(50, 36), covariance="spherical", corr_length=(0.2, 0.05, -0.05, 0.15),
                       anisotropy="geometric", approximate=True),
    "2d-gauss-geo": dict(dim=2, cells=(48, 48), covariance="gaussian", corr_length=(0.06, 0.0, 0.0, 0.04),
                         anisotropy="geometric"),
    "3d-matern32-axi": dict(dim=3, cells=(32, 24, 20), covariance="matern32", corr_length=(0.2, 0.1, 0.05),
                            anisotropy="axiparallel", approximate=True),
    "3d-exp-geo": dict(dim=3, cells=(24, 20, 16), covariance="exponential",
                       corr_length=(0.15, 0.02, 0.0, -0.03, 0.08, 0.01, 0.0, 0.02, 0.04), anisotropy="geometric",
                       approximate=True),
    "3d-gexp-iso-notransp": dict(dim=3, cells=(16, 20, 24), covariance="gammaExponential", exp_gamma=1.3,
                                 corr_length=0.1, transposed=0),
    "2d-matern-geo": dict(dim=2, cells=(40, 32), covariance="matern", matern_nu=1.7,
                          corr_length=(0.1, 0.02, -0.01, 0.06), anisotropy="geometric", approximate=True),
    "3d-matern-iso": dict(dim=3, cells=(20, 16, 12), covariance="matern", matern_nu=0.35, corr_length=0.1),
    # power-of-two tori: the FP32 schedules take the paired-FP32 (FFMA2) passes
    "2d-exp-pow2": dict(dim=2, cells=(128, 64), covariance="exponential", corr_length=0.1),
    "2d-sph-geo-pow2": dict(dim=2, cells=(64, 128), covariance="spherical", corr_length=(0.2, 0.05, -0.05, 0.15),
                            anisotropy="geometric", approximate=True),
    "3d-matern32-axi-pow2": dict(dim=3, cells=(64, 64, 64), covariance="matern32", corr_length=(0.2, 0.1, 0.05),
                                 anisotropy="axiparallel", approximate=True),
    "3d-exp-geo-pow2": dict(dim=3, cells=(128, 64, 64), covariance="exponential",
                            corr_length=(0.15, 0.02, 0.0, -0.03, 0.08, 0.01, 0.0, 0.02, 0.04),
                            anisotropy="geometric", approximate=True),
    "3d-exp-iso-notransp-pow2": dict(dim=3, cells=(64, 64, 128), covariance="exponential", corr_length=0.05,
                                     transposed=0),
    # 3-smooth tori (96, 192, 384, 768): the fast scalar kernels with a radix-3 stage
    "3d-matern32-3smooth": dict(dim=3, cells=(48, 96, 192), covariance="matern32", corr_length=0.1,
                                approximate=True),
    "2d-exp-geo-3smooth": dict(dim=2, cells=(384, 96), covariance="exponential",
                               corr_length=(0.1, 0.02, -0.02, 0.05), anisotropy="geometric", approximate=True),
    # 5-smooth tori (160, 320, 640): radix-5 stages of the generic kernels
    "3d-exp-5smooth": dict(dim=3, cells=(80, 160, 320), covariance="exponential", corr_length=0.08,
                           approximate=True),
    # merge periodization (matrix.hh:652-775): radial branch needs sqrt(dim) < factor/2
    "2d-merge-radialplus-f3": dict(dim=2, cells=(48, 40), covariance="matern32", corr_length=0.3,
                                   embedding_factor=3, periodization="merge", sigmoid_start=1.0,
                                   sigmoid_end=2.0, approximate=True),
    "3d-merge-tensor-smooth": dict(dim=3, cells=(16, 16, 12), covariance="exponential", corr_length=0.2,
                                   periodization="merge", sigmoid="smooth", sigmoid_combine="tensor",
                                   sigmoid_start=0.7, sigmoid_end=1.0, approximate=True),
    "2d-merge-radial-geo-f4": dict(dim=2, cells=(32, 24), covariance="exponential",
                                   corr_length=(0.2, 0.05, -0.05, 0.15), anisotropy="geometric",
                                   embedding_factor=4, periodization="merge", sigmoid_combine="radial",
                                   sigmoid_start=1.0, sigmoid_end=3.0, approximate=True),
    # fold periodization (matrix.hh:791-890)
    "2d-fold-smoothstep-f3": dict(dim=2, cells=(48, 40), covariance="exponential", corr_length=0.3,
                                  embedding_factor=3, periodization="fold", approximate=True),
    "3d-fold-smooth": dict(dim=3, cells=(16, 16, 12), covariance="matern32", corr_length=(0.2, 0.1, 0.1),
                           anisotropy="axiparallel", periodization="fold", sigmoid="smooth",
                           fold_max_factor=2.0, approximate=True),
    # cofold periodization (matrix.hh:905-1013): DCT matrix (iso / axiparallel) and R2C (geometric)
    "2d-cofold-smoothstep-f3": dict(dim=2, cells=(48, 40), covariance="exponential", corr_length=0.3,
                                    embedding_factor=3, periodization="cofold", approximate=True),
    "3d-cofold-smooth-f4": dict(dim=3, cells=(16, 12, 12), covariance="matern32", corr_length=0.25,
                                embedding_factor=4, periodization="cofold", sigmoid="smooth",
                                cofold_max_factor=3.0, approximate=True),
    "2d-cofold-geo-r2c-f4": dict(dim=2, cells=(24, 20), covariance="exponential",
                                 corr_length=(0.4, 0.1, -0.1, 0.3), anisotropy="geometric", embedding_factor=4,
                                 periodization="cofold", cofold_recursions=3, approximate=True),
    # the remaining covariance functors (covariance.hh:465-489, 633-744, 799-823)
    "2d-sepexp-axi": dict(dim=2, cells=(48, 40), covariance="separableExponential", corr_length=(0.1, 0.2),
                          anisotropy="axiparallel"),
    "3d-sepexp-iso": dict(dim=3, cells=(16, 20, 12), covariance="separableExponential", corr_length=0.1),
    "2d-damped-iso": dict(dim=2, cells=(48, 40), covariance="dampedOscillation", corr_length=0.1),
    "3d-damped-geo": dict(dim=3, cells=(16, 12, 12), covariance="dampedOscillation",
                          corr_length=(0.1, 0.02, 0.0, -0.02, 0.08, 0.0, 0.0, 0.0, 0.05), anisotropy="geometric"),
    "2d-cauchy-geo": dict(dim=2, cells=(40, 32), covariance="cauchy", corr_length=(0.1, 0.02, -0.01, 0.06),
                          anisotropy="geometric"),
    "3d-cauchy-iso": dict(dim=3, cells=(16, 16, 12), covariance="cauchy", corr_length=0.08),
    "2d-gcauchy-axi": dict(dim=2, cells=(40, 48), covariance="generalizedCauchy", cauchy_alpha=1.5, cauchy_beta=0.8,
                           corr_length=(0.1, 0.05), anisotropy="axiparallel", approximate=True),
    "3d-gcauchy-iso": dict(dim=3, cells=(12, 16, 20), covariance="generalizedCauchy", cauchy_alpha=0.7,
                           cauchy_beta=2.5, corr_length=0.1),
    "2d-white-iso": dict(dim=2, cells=(40, 36), covariance="whiteNoise", corr_length=0.1),
    "3d-white-iso": dict(dim=3, cells=(12, 10, 8), covariance="whiteNoise", corr_length=0.1),
    # tori whose lengths have prime factors above 13: Bluestein transforms
    "2d-exp-prime": dict(dim=2, cells=(131, 97), covariance="exponential", corr_length=0.1),
    "3d-sph-prime": dict(dim=3, cells=(17, 19, 23), covariance="spherical", corr_length=0.2),
    "2d-exp-geo-prime-long": dict(dim=2, cells=(64, 2039), covariance="exponential",
                                  corr_length=(0.1, 0.02, -0.02, 0.05), anisotropy="geometric", approximate=True),
}


def plan_and_oracle(oracle, cfg, **over):
    d = desc_of(cfg, **over)
    P = pfb200.Plan(d)
    lam, st, status = oracle.spectrum(d)
    return d, P, lam, st, status


@pytest.mark.parametrize("name", list(CONFIGS))
def test_spectrum_and_stats(oracle, name):
    d, P, lam, st, status = plan_and_oracle(oracle, CONFIGS[name])
    assert status == 0  # configs with negative eigenvalues set embedding.approximate
    gst = P.spectrum_build()
    glam = P.spectrum()
    assert rel(glam, lam) < TOL64
    assert (gst["small"], gst["zero"], gst["negative"]) == (st["small"], st["zero"], st["negative"])
    assert abs(gst["smallest"] - st["smallest"]) <= 1e-12 * max(abs(st["smallest"]), 1e-300) + 1e-18


def test_reference_eigen_scan_mode(oracle):
    cfg = dict(dim=2, cells=(32, 32), covariance="gaussian", corr_length=(0.5, 0.0, 0.0, 0.5),
               anisotropy="geometric", approximate=True)
    for mode in (pfb200.EIGCHECK_CORRECTED, pfb200.EIGCHECK_REFERENCE):
        d, P, lam, st, _ = plan_and_oracle(oracle, cfg, eigen_check=mode)
        gst = P.spectrum_build()
        assert (gst["small"], gst["zero"], gst["negative"]) == (st["small"], st["zero"], st["negative"])
        assert rel(P.spectrum(), lam) < TOL64


def test_negative_eigenvalues_raise(oracle):
    cfg = dict(dim=2, cells=(32, 32), covariance="gaussian", corr_length=0.5)
    P = pfb200.Plan(desc_of(cfg))
    with pytest.raises(pfb200.NegativeEigenvalueError, match="negative eigenvalues"):
        P.spectrum_build()


@pytest.mark.parametrize("prec", [pfb200.PREC_F64, pfb200.PREC_F32])
@pytest.mark.parametrize("name", list(CONFIGS))
def test_generate_parity(oracle, name, prec):
    d, P, lam, st, _ = plan_and_oracle(oracle, CONFIGS[name], precision=prec)
    g = oracle.resolve(d)
    noise = oracle.noise(20261203, g.noise)
    ref, _ = oracle.generate(d, lam, noise)
    out = P.generate(noise=noise)
    assert rel(out, ref) < (TOL64F if prec == pfb200.PREC_F64 else TOL32)


@pytest.mark.parametrize("prec", [pfb200.PREC_F64, pfb200.PREC_F32])
@pytest.mark.parametrize("op", [pfb200.OP_MUL, pfb200.OP_ROOT, pfb200.OP_INVEXT])
@pytest.mark.parametrize("name", ["2d-exp-iso", "2d-sph-geo", "3d-gexp-iso-notransp", "3d-exp-geo",
                                  "3d-matern32-axi", "2d-exp-prime", "3d-sph-prime",
                                  "2d-sepexp-axi", "3d-damped-geo", "2d-cauchy-geo", "3d-gcauchy-iso",
                                  "2d-white-iso",
                                  # power-of-two tori: FP32 takes the paired fused pass
                                  "2d-exp-pow2", "3d-matern32-axi-pow2", "3d-exp-geo-pow2"])
def test_matvec_parity(oracle, name, op, prec):
    d, P, lam, st, _ = plan_and_oracle(oracle, CONFIGS[name])
    if op == pfb200.OP_INVEXT and (lam <= 0).any():
        pytest.skip("clamped zero eigenvalues: 1/lambda is infinite in the reference too")
    g = oracle.resolve(d)
    x = np.random.default_rng(5).standard_normal(g.domain)
    ref = oracle.matvec(d, lam, op, x)
    dt = np.float64 if prec == pfb200.PREC_F64 else np.float32
    out = P.matvec(x.astype(dt), op=op, precision=prec)
    assert rel(out, ref) < (TOL64 if prec == pfb200.PREC_F64 else TOL32)


@pytest.mark.parametrize("name", ["2d-exp-iso", "3d-gexp-iso-notransp", "2d-cubic-axi"])
def test_cg_reference_mode(oracle, name):
    """innerCG with the reference's stopping rules.  Its energy-stagnation test
    (|E_k - E_{k-1}| / |E_k - E_0| < 1e-16, matrix.hh:1422-1425) fires once the energy
    stops changing in the last bit, which depends on the summation order of the FP64
    dot products, so the iteration count may differ after stagnation; the solutions
    must agree and both must have reached the stagnation level."""
    d, P, lam, st, _ = plan_and_oracle(oracle, CONFIGS[name], cg_iterations=60)
    g = oracle.resolve(d)
    b = np.random.default_rng(9).standard_normal(g.domain)
    xo, its = oracle.multiply_inverse(d, lam, b)
    x, rep = P.multiply_inverse(b, mode=pfb200.CG_REFERENCE)
    assert rep["iterations"] > 0 and its > 0
    assert rel(x, xo) < 1e-8
    r_gpu = rel(oracle.matvec(d, lam, pfb200.OP_MUL, x), b)
    r_orc = rel(oracle.matvec(d, lam, pfb200.OP_MUL, xo), b)
    # same algorithm, same quality: either both stop far from convergence (the compactly
    # supported cubic covariance within 60 iterations) or both stop on the stagnation rule
    # once the residual is tiny (where the last FP64 bits decide the exact iteration)
    assert r_gpu <= max(1.01 * r_orc, 1e-7)
    assert abs(rep["relative_residual"] - r_gpu) <= 1e-3 * r_gpu + 1e-14


@pytest.mark.parametrize("name", ["3d-gexp-iso-notransp", "3d-matern32-axi", "2d-sph-geo"])
@pytest.mark.parametrize("inner_fp32", [False, True])
def test_cg_residual_mode(oracle, inner_fp32, name):
    """True-residual mode reaches 1e-8 also where clamped eigenvalues make the torus
    inverse singular (the preconditioner then uses the pseudo-inverse)."""
    d, P, lam, st, _ = plan_and_oracle(oracle, CONFIGS[name])
    g = oracle.resolve(d)
    b = np.random.default_rng(11).standard_normal(g.domain)
    x, rep = P.multiply_inverse(b, mode=pfb200.CG_RESIDUAL, tolerance=1e-8, inner_fp32=inner_fp32)
    assert rep["relative_residual"] <= 1e-8
    # the oracle's FP64 matvec confirms the residual
    assert rel(oracle.matvec(d, lam, pfb200.OP_MUL, x), b) <= 1.1e-8


def test_cg_zero_rhs():
    P = pfb200.Plan(desc_of(CONFIGS["2d-exp-iso"]))
    b = np.zeros(64 * 48)
    x, rep = P.multiply_inverse(b)
    assert rep["iterations"] == 0 and not x.any()


@pytest.mark.parametrize("kind", ["logNormal", "foldedNormal", "sign", "boxCox"])
def test_generate_with_transform(oracle, kind):
    cfg = dict(CONFIGS["2d-exp-iso"], transform=kind, boxcox_lambda=0.2)
    d, P, lam, st, _ = plan_and_oracle(oracle, cfg)
    g = oracle.resolve(d)
    noise = oracle.noise(3, g.noise)
    ref, _ = oracle.generate(d, lam, noise)
    ref = oracle.transform(kind, ref, boxcox_lambda=0.2)
    out = P.generate(noise=noise, apply_transform=True)
    if kind == "sign":
        assert (out == ref).mean() > 0.999
    else:
        assert rel(out, ref) < 1e-11
    v = np.random.default_rng(4).standard_normal(1000) * 0.3
    np.testing.assert_allclose(P.apply_transform(v.copy()), oracle.transform(kind, v, boxcox_lambda=0.2),
                               rtol=1e-13)


def test_1d_dft_backend_and_spare_field(oracle):
    cfg = dict(dim=1, cells=(96,), covariance="exponential", corr_length=0.05)
    d, P, lam, st, _ = plan_and_oracle(oracle, cfg)
    assert P.info.matrix_backend == pfb200.MATRIX_DFT and P.info.field_backend == pfb200.FIELD_DFT
    g = oracle.resolve(d)
    noise = oracle.noise(1, g.noise)
    ref, spare = oracle.generate(d, lam, noise)
    out1 = P.generate(noise=noise)
    out2 = P.generate(noise=oracle.noise(2, g.noise))  # returns the cached second field
    assert rel(P.spectrum(), lam) < TOL64
    assert rel(out1, ref) < TOL64 and rel(out2, spare) < TOL64
    x = np.random.default_rng(3).standard_normal(g.domain)
    assert rel(P.matvec(x), oracle.matvec(d, lam, pfb200.OP_MUL, x)) < TOL64


@pytest.mark.parametrize("dim", [2, 3])
def test_dft_matrix_and_field_backends(oracle, dim):
    cells = (24, 20) if dim == 2 else (12, 10, 8)
    cfg = dict(dim=dim, cells=cells, covariance="matern52", corr_length=0.15,
               matrix_backend=pfb200.MATRIX_DFT, field_backend=pfb200.FIELD_DFT)
    d, P, lam, st, _ = plan_and_oracle(oracle, cfg)
    g = oracle.resolve(d)
    P.spectrum_build()
    assert rel(P.spectrum(), lam) < TOL64
    noise = oracle.noise(5, g.noise)
    ref, spare = oracle.generate(d, lam, noise)
    assert rel(P.generate(noise=noise), ref) < TOL64
    assert rel(P.generate(noise=noise), spare) < TOL64
    x = np.random.default_rng(3).standard_normal(g.domain)
    for op in (pfb200.OP_MUL, pfb200.OP_ROOT, pfb200.OP_INVEXT):
        assert rel(P.matvec(x, op=op), oracle.matvec(d, lam, op, x)) < TOL64


@pytest.mark.parametrize("dim", [2, 3])
def test_dft_matrix_with_r2c_field(oracle, dim):
    cells = (24, 20) if dim == 2 else (12, 10, 8)
    cfg = dict(dim=dim, cells=cells, covariance="matern52", corr_length=0.15,
               matrix_backend=pfb200.MATRIX_DFT, field_backend=pfb200.FIELD_R2C)
    d, P, lam, st, _ = plan_and_oracle(oracle, cfg)
    g = oracle.resolve(d)
    noise = oracle.noise(6, g.noise)
    ref, _ = oracle.generate(d, lam, noise)
    assert rel(P.generate(noise=noise), ref) < TOL64
    x = np.random.default_rng(4).standard_normal(g.domain)
    assert rel(P.matvec(x, op=pfb200.OP_ROOT), oracle.matvec(d, lam, pfb200.OP_ROOT, x)) < TOL64


def test_device_pointers(oracle):
    torch = pytest.importorskip("torch")
    d, P, lam, st, _ = plan_and_oracle(oracle, CONFIGS["3d-matern32-axi"], precision=pfb200.PREC_F32)
    g = oracle.resolve(d)
    noise = oracle.noise(8, g.noise)
    ref, _ = oracle.generate(d, lam, noise)
    nd = torch.from_numpy(noise).cuda()
    out = torch.empty(g.domain, dtype=torch.float32, device="cuda")
    P.generate(noise=nd, out=out)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), ref) < TOL32
    x = torch.randn(g.domain, dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    P.matvec(x, precision=pfb200.PREC_F32, out=y)
    torch.cuda.synchronize()
    assert rel(y.cpu().numpy(), oracle.matvec(d, lam, pfb200.OP_MUL, x.cpu().double().numpy())) < TOL32


def test_counter_based_noise_statistics(oracle):
    """Seeded on-device noise: the empirical covariance of many realizations matches the
    exact covariance of the reference's generator (J J^T, J = d field / d noise,
    computed with the oracle from unit noise vectors)."""
    cfg = dict(dim=2, cells=(8, 6), covariance="exponential", corr_length=0.3)
    d, P, lam, st, _ = plan_and_oracle(oracle, cfg)
    g = oracle.resolve(d)
    J = np.stack([oracle.generate(d, lam, np.eye(g.noise)[i])[0] for i in range(g.noise)], axis=1)
    exact = J @ J.T
    M = 20000
    fields = P.generate_batch(seed=123, count=M).reshape(M, g.domain)
    emp = fields.T @ fields / M
    se = np.sqrt((np.diag(exact)[:, None] * np.diag(exact)[None, :] + exact ** 2) / M)
    assert np.abs(fields.mean(axis=0)).max() < 5 * np.sqrt(np.diag(exact).max() / M)
    assert (np.abs(emp - exact) < 5 * se + 1e-12).mean() > 0.995


@pytest.mark.parametrize("prec", [pfb200.PREC_F64, pfb200.PREC_F32])
@pytest.mark.parametrize("name", ["2d-exp-pow2", "2d-sph-geo-pow2", "3d-matern32-axi-pow2",
                                  "3d-exp-iso-notransp-pow2", "2d-exp-iso", "3d-matern32-axi"])
def test_counter_noise_matches_host_philox(oracle, name, prec):
    """generate(seed) equals the oracle fed the host reproduction of the counter-based
    noise: checks the counter layout, the (k, k + T/2) pairing, the self-conjugate rule and
    the transforms of the seeded path (fast-intrinsic Box-Muller: ~1e-6 per normal)."""
    d, P, lam, st, _ = plan_and_oracle(oracle, CONFIGS[name], precision=prec)
    g = oracle.resolve(d)
    seed = 0x1234ABCD5678
    ref, _ = oracle.generate(d, lam, counter_noise(g, seed, prec == pfb200.PREC_F64))
    out = P.generate(seed=seed)
    assert rel(out, ref) < (1e-9 if prec == pfb200.PREC_F64 else TOL32)


# ---------------------------------------------------------------------------
# ensembles: fields of different sizes and covariances from one captured graph
# ---------------------------------------------------------------------------
ENSEMBLE = [
    dict(dim=2, cells=(131, 97), covariance="exponential", corr_length=(0.1, 0.03, -0.02, 0.06),
         anisotropy="geometric", approximate=True),
    dict(dim=2, cells=(128, 256), covariance="gaussian", corr_length=(0.05, 0.0, 0.0, 0.05),
         anisotropy="geometric", approximate=True),
    dict(dim=2, cells=(200, 150), covariance="spherical", corr_length=(0.2, 0.1, -0.1, 0.15),
         anisotropy="geometric", approximate=True),
    dict(dim=2, cells=(64, 64), covariance="cubic", corr_length=(0.3, 0.0, 0.0, 0.3),
         anisotropy="geometric", approximate=True),
    dict(dim=3, cells=(32, 24, 20), covariance="matern32", corr_length=(0.2, 0.1, 0.05),
         anisotropy="axiparallel", approximate=True),
]


def test_ensemble_matches_single_field_oracle(oracle):
    """Every field of two successive ensemble calls equals the oracle fed the host
    reproduction of its counter-based noise (seed + i, epoch = call number)."""
    descs = [desc_of(c, precision=pfb200.PREC_F32) for c in ENSEMBLE]
    E = pfb200.Ensemble(descs, seed=777)
    stats = E.spectra()
    for call in (1, 2):
        out = E.generate()
        assert E.launches_per_replay() > len(descs)
        for i, d in enumerate(descs):
            g = oracle.resolve(d)
            lam, ost, _ = oracle.spectrum(d)
            assert stats[i]["negative"] == ost["negative"]
            ref, _ = oracle.generate(d, lam, counter_noise(g, 777 + i, False, epoch=call))
            assert rel(E.field(out, i), ref) < TOL32, (call, i)
    E.close()


def test_ensemble_autotune_keeps_parity(oracle):
    """Measured planning of every field changes kernel choices only: after it (and a new
    capture) each field still equals the oracle on its reproduced counters."""
    pfb200.wisdom_forget()
    descs = [desc_of(c, precision=pfb200.PREC_F32) for c in ENSEMBLE[:4]]
    E = pfb200.Ensemble(descs, seed=99)
    E.spectra()
    E.generate()  # captured before tuning: the tuner drops this graph
    assert E.autotune(repetitions=1) == len(descs)
    out = E.generate()  # call 2 of this ensemble
    for i, d in enumerate(descs):
        g = oracle.resolve(d)
        lam, _, _ = oracle.spectrum(d)
        ref, _ = oracle.generate(d, lam, counter_noise(g, 99 + i, False, epoch=2))
        assert rel(E.field(out, i), ref) < TOL32, i
    E.close()
    pfb200.wisdom_forget()


def test_ensemble_device_replay_is_new_noise(oracle):
    torch = pytest.importorskip("torch")
    descs = [desc_of(c, precision=pfb200.PREC_F32) for c in ENSEMBLE[:3]]
    E = pfb200.Ensemble(descs, seed=5)
    E.spectra()
    a = torch.empty(E.total, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    E.generate(a)
    E.generate(b)
    torch.cuda.synchronize()
    assert not torch.equal(a, b)
    assert abs(float(a.std()) - float(b.std())) < 0.2 * float(a.std())
    E.close()


# ---------------------------------------------------------------------------
# DCT/DST field backend (opt-in in the reference; fftw.transposed = false)
# ---------------------------------------------------------------------------
DCTDST = {
    "2d-exp-iso": dict(dim=2, cells=(40, 36), covariance="exponential", corr_length=0.1),
    "2d-m52-axi-pow2": dict(dim=2, cells=(128, 64), covariance="matern52", corr_length=(0.1, 0.05),
                            anisotropy="axiparallel", approximate=True),
    "3d-sph-iso": dict(dim=3, cells=(20, 16, 12), covariance="spherical", corr_length=0.2),
}


def _dctdst_descs(cfg, prec, **extra):
    over = dict(transposed=0, precision=prec, matrix_backend=pfb200.MATRIX_DCT, **extra)
    return (desc_of(cfg, field_backend=pfb200.FIELD_DCTDST, **over),
            desc_of(cfg, field_backend=pfb200.FIELD_R2C, **over))


@pytest.mark.parametrize("prec", [pfb200.PREC_F64, pfb200.PREC_F32])
@pytest.mark.parametrize("name", list(DCTDST))
def test_dctdst_generate_parity(oracle, name, prec):
    d, dr = _dctdst_descs(DCTDST[name], prec, transform="logNormal")
    lam, st, _ = oracle.spectrum(dr)
    P = pfb200.Plan(d)
    P.spectrum_build()
    assert P.info.noise_size == oracle.dctdst_noise_size(d)
    noise = oracle.noise(20261203, P.info.noise_size)
    tol = TOL64F if prec == pfb200.PREC_F64 else TOL32
    ref = oracle.generate_dctdst(d, lam, noise)
    assert rel(P.generate(noise=noise), ref) < tol
    # the value transform acts on the summed field of all symmetry types
    assert rel(P.generate(noise=noise, apply_transform=True), np.exp(ref)) < tol
    P.close()


def test_dctdst_seeded_covariance(oracle):
    """Seeded DCT/DST realizations: empirical covariance against the exact covariance of the
    circulant embedding (which the DCT/DST generator reproduces exactly)."""
    cfg = dict(dim=2, cells=(8, 6), covariance="exponential", corr_length=0.3)
    d, dr = _dctdst_descs(cfg, pfb200.PREC_F64)
    lam, _, _ = oracle.spectrum(dr)
    g = oracle.resolve(dr)
    C = np.stack([oracle.matvec(dr, lam, pfb200.OP_MUL, np.eye(g.domain)[j]) for j in range(g.domain)], axis=1) * g.N
    P = pfb200.Plan(d)
    M = 20000
    fields = P.generate_batch(seed=99, count=M).reshape(M, g.domain)
    emp = fields.T @ fields / M
    se = np.sqrt((np.diag(C)[:, None] * np.diag(C)[None, :] + C ** 2) / M)
    assert (np.abs(emp - C) < 5 * se + 1e-12).mean() > 0.995
    P.close()


@pytest.mark.parametrize("prec", [pfb200.PREC_F64, pfb200.PREC_F32])
@pytest.mark.parametrize("name", list(DCTDST))
def test_dctdst_matvec_parity(oracle, name, prec):
    """Products of the DCT/DST field backend (matrix.hh:1449-1473, one r2r product per
    symmetry type, summed) equal the circulant product (C_ext x)/N on the domain, which the
    oracle computes through the R2C field backend with the same DCT eigenvalues."""
    d, dr = _dctdst_descs(DCTDST[name], prec)
    lam, _, _ = oracle.spectrum(dr)
    g = oracle.resolve(dr)
    P = pfb200.Plan(d)
    P.spectrum_build()
    x = np.random.default_rng(8).standard_normal(g.domain)
    dt = np.float64 if prec == pfb200.PREC_F64 else np.float32
    for op in (pfb200.OP_MUL, pfb200.OP_ROOT, pfb200.OP_INVEXT):
        # 1/lambda amplifies the rounding of tiny eigenvalues (condition number of the torus)
        if op == pfb200.OP_INVEXT and lam.min() < 1e-6 * lam.max():
            continue
        out = P.matvec(x.astype(dt), op=op, precision=prec)
        assert rel(out, oracle.matvec(dr, lam, op, x)) < (TOL64 if prec == pfb200.PREC_F64 else TOL32), op
    if name == "2d-exp-iso":
        # CG on the DCT/DST plan: the same operator, so the residual-mode solve converges
        b = np.random.default_rng(9).standard_normal(g.domain)
        xs, rep = P.multiply_inverse(b, mode=pfb200.CG_RESIDUAL, tolerance=1e-8)
        assert rep["relative_residual"] <= 1e-8
        assert rel(oracle.matvec(dr, lam, pfb200.OP_MUL, xs), b) <= 1.1e-8
    P.close()


@pytest.mark.parametrize("name", list(DCTDST))
def test_dctdst_transposed_draw_order(oracle, name):
    """The reference's default fftw.transposed (dim > 1): the draws of each symmetry type
    follow the field backend's local cells with the last two dimensions swapped
    (dctdstfieldbackend.hh:855-871, matrix.hh:349-360); buffered noise and seeded
    generation against the oracle, whose eigenvalues are taken in the natural layout."""
    d = desc_of(DCTDST[name], field_backend=pfb200.FIELD_DCTDST, matrix_backend=pfb200.MATRIX_DCT)
    dr = desc_of(DCTDST[name], field_backend=pfb200.FIELD_R2C, matrix_backend=pfb200.MATRIX_DCT, transposed=0)
    lam, _, _ = oracle.spectrum(dr)
    P = pfb200.Plan(d)
    assert P.info.transposed == 1
    P.spectrum_build()
    noise = oracle.noise(11, P.info.noise_size)
    assert rel(P.generate(noise=noise), oracle.generate_dctdst(d, lam, noise)) < TOL64F
    # the untransposed plan on the same buffer gives a different field (another draw order)
    Pn = pfb200.Plan(desc_of(DCTDST[name], field_backend=pfb200.FIELD_DCTDST, matrix_backend=pfb200.MATRIX_DCT,
                             transposed=0))
    assert rel(Pn.generate(noise=noise), oracle.generate_dctdst(d, lam, noise)) > 1e-3
    P.close()
    Pn.close()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("name", ["3d-matern32-axi-pow2", "2d-exp-prime"])
def test_pipelined_batch_equals_single_calls(name, mode):
    """pf_generate_batch with device output alternates realizations over two streams with
    separate workspaces; every realization equals the one-at-a-time call with its seed."""
    torch = pytest.importorskip("torch")
    d = desc_of(CONFIGS[name], precision=pfb200.PREC_F32)
    P = pfb200.Plan(d)
    pfb200.wisdom_forget()
    P.autotune(repetitions=1)
    lines = [l.split() for l in pfb200.wisdom_export().strip().splitlines()]
    for f in lines:
        if f[0] == "3":
            f[5] = str(mode)
    pfb200.wisdom_forget()
    pfb200.wisdom_import("\n".join(" ".join(f) for f in lines) + "\n")
    P.close()
    P = pfb200.Plan(d)
    assert P.autotune() is False  # choices and batch mode from the wisdom
    pfb200.wisdom_forget()
    n = P.info.domain_size
    batch = torch.empty(5 * n, dtype=torch.float32, device="cuda")
    P.generate_batch(seed=41, count=5, out=batch)
    one = torch.empty(n, dtype=torch.float32, device="cuda")
    for r in range(5):
        P.generate(seed=41 + r, out=one)
        torch.cuda.synchronize()
        assert torch.equal(batch[r * n:(r + 1) * n], one), r
    P.close()


@pytest.mark.parametrize("name", ["3d-matern32-axi-pow2", "2d-exp-prime"])
def test_autotune_and_wisdom(oracle, name):
    """Measured planning changes only kernel choices: parity holds after it; the wisdom it
    records serves a second plan without timing, also after an export/import round trip."""
    pfb200.wisdom_forget()
    d, P, lam, st, _ = plan_and_oracle(oracle, CONFIGS[name], precision=pfb200.PREC_F32)
    g = oracle.resolve(d)
    noise = oracle.noise(7, g.noise)
    ref, _ = oracle.generate(d, lam, noise)
    assert P.autotune(repetitions=2) is True
    assert rel(P.generate(noise=noise), ref) < TOL32
    text = pfb200.wisdom_export()
    assert len(text.strip().splitlines()) == g.dim + 1  # the passes and the batch mode
    P2 = pfb200.Plan(d)
    assert P2.autotune() is False
    pfb200.wisdom_forget()
    pfb200.wisdom_import(text)
    P3 = pfb200.Plan(d)
    assert P3.autotune() is False
    assert rel(P3.generate(noise=noise), ref) < TOL32
    pfb200.wisdom_forget()
    for Q in (P, P2, P3):
        Q.close()


def test_pipelined_batch_to_host_equals_device_batch():
    torch = pytest.importorskip("torch")
    P = pfb200.Plan(desc_of(CONFIGS["3d-matern32-axi-pow2"], precision=pfb200.PREC_F32))
    n = P.info.domain_size
    dev = torch.empty(4 * n, dtype=torch.float32, device="cuda")
    P.generate_batch(seed=9, count=4, out=dev)
    host = torch.empty(4 * n, dtype=torch.float32).pin_memory().numpy()
    P.generate_batch(seed=9, count=4, out=host)
    assert np.array_equal(host, dev.cpu().numpy())
    P.close()


@pytest.mark.parametrize("lanes", [1, 3])
@pytest.mark.parametrize("mode", [pfb200.CG_REFERENCE, pfb200.CG_RESIDUAL])
def test_cg_batch_lanes_equal_single_solves(oracle, mode, lanes):
    """pf_multiply_inverse_batch: every right-hand side gets the solution and report of a
    single pf_multiply_inverse call (same deterministic reductions), whichever lane runs
    it; host and device buffers."""
    torch = pytest.importorskip("torch")
    # reference mode starts from the torus inverse 1/lambda, which is infinite where the
    # clamped configurations have zero eigenvalues (in the reference too): a config without
    name = "3d-gexp-iso-notransp" if mode == pfb200.CG_REFERENCE else "3d-matern32-axi"
    d, P, lam, st, _ = plan_and_oracle(oracle, CONFIGS[name], cg_iterations=80)
    g = oracle.resolve(d)
    B = np.random.default_rng(21).standard_normal((5, g.domain))
    B[2] = 0.0  # the zero-field shortcut inside a batch
    kw = dict(mode=mode, tolerance=1e-8, inner_fp32=True)
    singles = [P.multiply_inverse(B[i], **kw) for i in range(5)]
    X, reps = P.multiply_inverse_batch(B, lanes=lanes, **kw)
    for i in range(5):
        assert rel(X[i], singles[i][0]) <= 1e-14 if B[i].any() else not X[i].any(), i
        assert reps[i]["iterations"] == singles[i][1]["iterations"], i
    if mode == pfb200.CG_RESIDUAL:
        assert max(r["relative_residual"] for r in reps) <= 1e-8
    Bd = torch.from_numpy(B).cuda()
    Xd = torch.empty_like(Bd)
    P.multiply_inverse_batch(Bd, Xd, lanes=lanes, **kw)
    torch.cuda.synchronize()
    assert rel(Xd.cpu().numpy(), X) <= 1e-14
    P.close()
