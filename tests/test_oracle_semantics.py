"""The FP64 oracle against an independent numpy/scipy restatement and against the
analytic properties of circulant embedding (matrix.hh:223-421, 1315-1646)."""
import numpy as np
import pytest

import npref
import pfb200
from helpers import desc_of, full_lambda, rel

CASES_2D = [
    dict(dim=2, cells=(16, 12), covariance=c, corr_length=0.15, anisotropy="none")
    for c in ["exponential", "gaussian", "spherical", "separableExponential", "matern32", "matern52",
              "dampedOscillation", "cauchy", "cubic", "whiteNoise"]
] + [
    dict(dim=2, cells=(16, 12), covariance="gammaExponential", exp_gamma=1.5, corr_length=0.15),
    dict(dim=2, cells=(16, 12), covariance="matern", matern_nu=0.8, corr_length=0.15),
    dict(dim=2, cells=(16, 12), covariance="matern", matern_nu=2.7, corr_length=0.1, approximate=True),
    dict(dim=2, cells=(16, 12), covariance="generalizedCauchy", cauchy_alpha=1.2, cauchy_beta=2.0,
         corr_length=0.15),
    dict(dim=2, cells=(20, 14), covariance="exponential", corr_length=(0.2, 0.07), anisotropy="axiparallel",
         extensions=(2.0, 1.0)),
    dict(dim=2, cells=(18, 16), covariance="matern52", corr_length=(0.2, 0.05, -0.03, 0.1),
         anisotropy="geometric", approximate=True),
]
CASES_3D = [
    dict(dim=3, cells=(8, 6, 10), covariance=c, corr_length=(0.2, 0.1, 0.15), anisotropy="axiparallel")
    for c in ["exponential", "matern32", "spherical", "gaussian"]
] + [
    dict(dim=3, cells=(8, 6, 10), covariance="matern", matern_nu=1.3, corr_length=(0.2, 0.1, 0.15),
         anisotropy="axiparallel", approximate=True),
    dict(dim=3, cells=(8, 6, 10), covariance="exponential",
         corr_length=(0.15, 0.02, 0.0, -0.03, 0.1, 0.01, 0.0, 0.02, 0.12), anisotropy="geometric",
         approximate=True),
]


@pytest.mark.parametrize("cfg", CASES_2D + CASES_3D, ids=lambda c: f"{c['dim']}d-{c['covariance']}-{c.get('anisotropy')}")
def test_spectrum_matches_numpy(oracle, cfg):
    d = desc_of(cfg)
    g = oracle.resolve(d)
    lam, stats, st = oracle.spectrum(d)
    ref = npref.spectrum_full(cfg)
    ref_clamped = np.where(ref < 0, 0.0, ref)
    got = full_lambda(g, lam)
    assert np.abs(got - ref_clamped).max() <= 1e-12 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("transposed", [-1, 0])
@pytest.mark.parametrize("cfg", CASES_2D[:3] + CASES_3D[:2] + [CASES_2D[-1], CASES_3D[-1]],
                         ids=lambda c: f"{c['dim']}d-{c['covariance']}-{c.get('anisotropy')}")
def test_generate_matches_numpy(oracle, cfg, transposed):
    d = desc_of(cfg, transposed=transposed)
    g = oracle.resolve(d)
    lam, stats, st = oracle.spectrum(d)
    noise = oracle.noise(7, g.noise)
    field, _ = oracle.generate(d, lam, noise)
    ref = npref.generate_r2c(cfg, full_lambda(g, lam), noise, bool(g.transposed))
    assert rel(field, ref) < 1e-12


@pytest.mark.parametrize("op", [pfb200.OP_MUL, pfb200.OP_ROOT, pfb200.OP_INVEXT])
@pytest.mark.parametrize("cfg", [CASES_2D[0], CASES_2D[-2], CASES_3D[0], CASES_3D[-1]],
                         ids=lambda c: f"{c['dim']}d-{c.get('anisotropy')}")
def test_matvec_matches_numpy(oracle, cfg, op):
    d = desc_of(cfg)
    g = oracle.resolve(d)
    lam, _, _ = oracle.spectrum(d)
    x = np.random.default_rng(1).standard_normal(g.domain)
    y = oracle.matvec(d, lam, op, x)
    shape = tuple(reversed(cfg["cells"][: cfg["dim"]]))
    ref = npref.matvec(cfg, full_lambda(g, lam), x.reshape(shape), op)
    assert rel(y, ref) < 1e-12


def test_eigenvalues_sum_to_variance(oracle):
    # classical embedding without clamping: sum_k lambda_k = c(0) = sigma^2
    cfg = dict(dim=2, cells=(32, 24), covariance="exponential", corr_length=0.1, variance=1.7)
    d = desc_of(cfg)
    g = oracle.resolve(d)
    lam, stats, st = oracle.spectrum(d)
    assert st == 0 and stats["negative"] == 0
    assert abs(full_lambda(g, lam).sum() - 1.7) < 1e-12


def test_unit_vector_matvec_is_scaled_covariance_column(oracle):
    # operator* returns (C x)/N (r2cmatrixbackend.hh:279-282 + r2cfieldbackend.hh:233-236)
    cfg = dict(dim=2, cells=(16, 12), covariance="gaussian", corr_length=0.2)
    d = desc_of(cfg)
    g = oracle.resolve(d)
    lam, _, _ = oracle.spectrum(d)
    x = np.zeros(g.domain)
    x[5 + 16 * 3] = 1.0
    y = oracle.matvec(d, lam, pfb200.OP_MUL, x).reshape(12, 16)
    c = npref.torus(cfg)
    ref = np.array([[c[(j1 - 3) % c.shape[0], (j0 - 5) % c.shape[1]] for j0 in range(16)] for j1 in range(12)])
    assert np.abs(y - ref / g.N).max() < 1e-15


def test_cg_inverse(oracle):
    cfg = dict(dim=2, cells=(16, 12), covariance="exponential", corr_length=0.1)
    d = desc_of(cfg)
    lam, _, _ = oracle.spectrum(d)
    b = np.random.default_rng(0).standard_normal(16 * 12)
    x, its = oracle.multiply_inverse(d, lam, b)
    assert 0 < its <= 100
    assert rel(oracle.matvec(d, lam, pfb200.OP_MUL, x), b) < 1e-8
    # zero right-hand side is returned unchanged (matrix.hh:193-205)
    z, its0 = oracle.multiply_inverse(d, lam, np.zeros(16 * 12))
    assert its0 == 0 and not z.any()


def test_reference_eigen_scan_defect(oracle):
    # R2C real-view scan (r2cmatrixbackend.hh:164-170, 378-400): only the first N_c
    # doubles (= N_c/2 complex entries) are checked; compare both modes with numpy
    cfg = dict(dim=2, cells=(16, 16), covariance="gaussian", corr_length=(0.5, 0.0, 0.0, 0.5),
               anisotropy="geometric", approximate=True)
    lam_c, st_c, _ = oracle.spectrum(desc_of(cfg, eigen_check=pfb200.EIGCHECK_CORRECTED))
    lam_r, st_r, _ = oracle.spectrum(desc_of(cfg, eigen_check=pfb200.EIGCHECK_REFERENCE))
    c = npref.torus(cfg)
    X = np.fft.rfftn(c) / c.size
    flat = X.ravel()
    re = flat.real
    assert st_c["negative"] == int((re <= -1e-14).sum()) and st_c["negative"] > 0
    view = np.stack([flat.real, flat.imag], axis=-1).ravel()[: flat.size]
    assert st_r["negative"] == int((view <= -1e-14).sum())
    assert st_r["smallest"] == view.min()
    # corrected mode clamps every negative real part; the reference mode leaves the
    # second half unclamped
    assert (lam_c >= 0).all()
    half = flat.size // 2
    assert (lam_r[half + 1:] < 0).any()
    np.testing.assert_allclose(lam_r[half + 1:], re[half + 1:], rtol=0, atol=1e-15)


def test_negative_eigenvalue_status(oracle):
    cfg = dict(dim=2, cells=(16, 16), covariance="gaussian", corr_length=0.5)
    _, st, status = oracle.spectrum(desc_of(cfg))
    assert st["negative"] > 0 and status == pfb200.PF_ERR_NEG_EIGEN
    _, _, status = oracle.spectrum(desc_of(cfg, approximate=True))
    assert status == 0


@pytest.mark.parametrize("kind", ["none", "logNormal", "foldedNormal", "sign", "boxCox"])
def test_value_transforms(oracle, kind):
    v = np.random.default_rng(2).standard_normal(1000) * 0.5
    out = oracle.transform(kind, v, boxcox_lambda=0.3)
    ref = {"none": v, "logNormal": np.exp(v), "foldedNormal": np.abs(v),
           "sign": np.where(v < 0, -1.0, 1.0), "boxCox": (v * 0.3 + 1) ** -0.3}[kind]
    np.testing.assert_allclose(out, ref, rtol=1e-15)


@pytest.mark.parametrize("over,msg", [
    (dict(dim=3, cells=(4, 4, 4), covariance="cubic", corr_length=0.1), "cubic"),
    (dict(covariance="gammaExponential", exp_gamma=2.5), "gamma"),
    (dict(covariance="generalizedCauchy", cauchy_alpha=3.0), "alpha"),
    (dict(covariance="matern", matern_nu=-1.0), "matern nu has to be positive"),
])
def test_config_errors(oracle, over, msg):
    cfg = dict(dim=2, cells=(8, 8), covariance="exponential", corr_length=0.1)
    cfg.update(over)
    with pytest.raises(ValueError, match=msg):
        oracle.resolve(desc_of(cfg))


def test_default_backends_and_layout(oracle):
    g = oracle.resolve(desc_of(dict(dim=2, cells=(8, 8), covariance="exponential", corr_length=0.1)))
    assert (g.matrix_backend, g.field_backend, g.transposed) == (pfb200.MATRIX_DCT, pfb200.FIELD_R2C, 0)
    g = oracle.resolve(desc_of(dict(dim=3, cells=(8, 6, 4), covariance="exponential", corr_length=0.1)))
    assert (g.matrix_backend, g.field_backend, g.transposed) == (pfb200.MATRIX_DCT, pfb200.FIELD_R2C, 1)
    assert list(g.Ts) == [16, 8, 12]
    g = oracle.resolve(desc_of(dict(dim=1, cells=(32,), covariance="exponential", corr_length=0.1)))
    assert (g.matrix_backend, g.field_backend, g.transposed) == (pfb200.MATRIX_DFT, pfb200.FIELD_DFT, 0)


@pytest.mark.parametrize("nu", [0.5, 1.5, 2.5])
def test_general_matern_matches_closed_forms(oracle, nu):
    """matern with nu = 1/2, 3/2, 5/2 equals exponential / matern32 / matern52 with the
    correlation length scaled by sqrt(2 nu) (covariance.hh:502-625)."""
    closed = {0.5: "exponential", 1.5: "matern32", 2.5: "matern52"}[nu]
    ell = 0.12
    a = desc_of(dict(dim=2, cells=(16, 12), covariance="matern", matern_nu=nu, corr_length=ell))
    b = desc_of(dict(dim=2, cells=(16, 12), covariance=closed, corr_length=ell))
    np.testing.assert_allclose(oracle.fill_matrix(a), oracle.fill_matrix(b), rtol=1e-12, atol=1e-15)


def test_dctdst_oracle_covariance_equals_circulant_embedding(oracle):
    """The DCT/DST restatement reproduces the embedded covariance: summing the 2^d symmetry
    types, the exact covariance J J^T of its generator equals the torus covariance restricted
    to the domain (circulant embedding without the R2C half-spectrum quirk)."""
    import pfb200
    d = pfb200.make_desc(dim=2, cells=(6, 5), covariance="exponential", corr_length=0.3, transposed=0,
                         field_backend=pfb200.FIELD_DCTDST)
    dr = pfb200.make_desc(dim=2, cells=(6, 5), covariance="exponential", corr_length=0.3, transposed=0)
    lam, st, _ = oracle.spectrum(dr)
    m = oracle.dctdst_noise_size(d)
    J = np.stack([oracle.generate_dctdst(d, lam, np.eye(m)[i]) for i in range(m)], axis=1)
    cov = J @ J.T
    # torus covariance between domain cells, from the unit-vector matvec (returns C e_j / N)
    g = oracle.resolve(dr)
    C = np.stack([oracle.matvec(dr, lam, pfb200.OP_MUL, np.eye(g.domain)[j]) for j in range(g.domain)], axis=1)
    C *= g.N
    assert np.abs(cov - C).max() < 1e-12 * np.abs(C).max()


def test_host_philox_known_answer():
    """The host reproduction of the device's counter-based generator (used to check seeded
    generation) is Philox4x32-10: known-answer vector for counter 0, key 0 (Salmon et al.)."""
    from helpers import _philox4x32_10
    z = np.zeros(1, dtype=np.uint64)
    assert [int(v[0]) for v in _philox4x32_10((z, z, z, z), 0)] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_merge_periodization_with_default_sigmoid_edges_is_classical(oracle):
    """embedding.periodization = merge with sigmoidStart 1 and sigmoidEnd = factor - 1 at
    factor 2 is a step at the domain extent: the merged torus covariance equals the classical
    mirroring (the two mirrors share the midpoint with weight 1/2 each)."""
    import pfb200
    for kw in (dict(dim=2, cells=(12, 10), covariance="matern32", corr_length=(0.2, 0.1)),
               dict(dim=3, cells=(6, 8, 4), covariance="exponential", corr_length=0.15)):
        for sig in ("smoothstep", "smooth"):
            base = pfb200.make_desc(**kw)
            merged = pfb200.make_desc(**kw, periodization="merge", sigmoid=sig)
            a, b = oracle.fill_matrix(base), oracle.fill_matrix(merged)
            assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()


def test_merge_periodization_smooths_the_embedding(oracle):
    """With factor 3 and a sigmoid transition between one and two extents, the merged
    covariance keeps the prescribed values on the domain (distances below one extent) and
    differs from the classical embedding in the transition zone."""
    import pfb200
    kw = dict(dim=2, cells=(16, 12), covariance="exponential", corr_length=0.5, embedding_factor=3)
    base = pfb200.make_desc(**kw)
    merged = pfb200.make_desc(**kw, periodization="merge", sigmoid_start=1.0, sigmoid_end=2.0,
                              sigmoid_combine="tensor")
    g = oracle.resolve(base)
    a = oracle.fill_matrix(base).reshape(g.T[1] // 2 + 1, g.T[0] // 2 + 1)
    b = oracle.fill_matrix(merged).reshape(g.T[1] // 2 + 1, g.T[0] // 2 + 1)
    inside = (np.arange(g.T[1] // 2 + 1)[:, None] < g.n[1]) & (np.arange(g.T[0] // 2 + 1)[None, :] < g.n[0])
    assert np.abs(a[inside] - b[inside]).max() < 1e-12
    assert np.abs(a[~inside] - b[~inside]).max() > 1e-6


def test_fold_periodization_keeps_domain_and_stretches_beyond(oracle):
    """embedding.periodization = fold (matrix.hh:791-890): within normalized radius 1 the
    covariance is the classical one; beyond it the radius r becomes 1 + int_1^r sigmoid, so
    the folded covariance at a cell equals the classical covariance at a shorter radius
    (never larger distance) and lies between the classical value and the value at radius 1."""
    import pfb200
    for sig in ("smoothstep", "smooth"):
        kw = dict(dim=2, cells=(16, 12), covariance="exponential", corr_length=0.5, embedding_factor=3)
        base = pfb200.make_desc(**kw)
        fold = pfb200.make_desc(**kw, periodization="fold", sigmoid=sig, fold_max_factor=1.0)
        g = oracle.resolve(base)
        a = oracle.fill_matrix(base).reshape(g.T[1] // 2 + 1, g.T[0] // 2 + 1)
        b = oracle.fill_matrix(fold).reshape(g.T[1] // 2 + 1, g.T[0] // 2 + 1)
        y, x = np.meshgrid(np.arange(g.T[1] // 2 + 1) * g.h[1], np.arange(g.T[0] // 2 + 1) * g.h[0], indexing="ij")
        r = np.sqrt((x ** 2 + y ** 2) / 2.0)
        inside = r <= 1.0
        assert np.abs(a[inside] - b[inside]).max() < 1e-14
        assert (b[~inside] >= a[~inside] - 1e-15).all()
        assert np.abs(a[~inside] - b[~inside]).max() > 1e-3


def _sigmoid_ref(kind, one, zero, x, rec):
    """SmoothstepSigmoid / SmoothSigmoid (covariance.hh:147-287), scalar restatement."""
    ax = abs(x)
    if kind == "smooth":
        if ax < one:
            return 1.0
        if ax > zero:
            return 0.0
        x1, x2 = (zero - ax) / (zero - one), (ax - one) / (zero - one)
        t1 = np.exp(-1.0 / x1) if x1 > 0 else 0.0
        t2 = np.exp(-1.0 / x2) if x2 > 0 else 0.0
        return t1 / (t1 + t2)
    x1 = 1.0 if ax < one else (0.0 if ax > zero else (zero - ax) / (zero - one))
    x2 = 2.0 * x1 - 1.0
    norm, add, out = 1.0, 1.0, 1.0
    for i in range(1, rec + 1):
        out *= 2.0 * i
        add *= 1 - x2 * x2
        out += add
        out /= 2.0 * i + 1.0
        norm *= 2.0 * i / (2.0 * i + 1.0)
    return (out * x2 / norm + 1.0) / 2.0


def _cofold_numpy(oracle, desc, base_values, sig, rec, max_factor):
    """modifyMatrixEntriesWithCofold (matrix.hh:905-1013) restated over the oracle's classical
    fill, with scipy's adaptive quadrature for the sigmoid integrals."""
    from scipy.integrate import quad
    import pfb200
    g = oracle.resolve(desc)
    if g.matrix_backend == pfb200.MATRIX_DCT:
        cells = [g.T[i] // 2 + 1 for i in range(g.dim)]
    elif g.matrix_backend == pfb200.MATRIX_R2C:
        cells = [2 * (g.T[0] // 2 + 1)] + [g.T[i] for i in range(1, g.dim)]
    else:
        cells = [g.T[i] for i in range(g.dim)]
    idx = np.arange(base_values.size)
    coords, r = [], idx.copy()
    for i in range(g.dim):
        c = (r % cells[i]).astype(np.float64) * g.h[i]
        r //= cells[i]
        half, wrap = 0.5 * g.ext[i] * g.factor, g.ext[i] * g.factor
        coords.append(np.where(c > half, c - wrap, c))
    norm = np.max(np.stack([np.abs(c) / g.ext[i] for i, c in enumerate(coords)]), axis=0)
    border = np.zeros(idx.size, bool)
    for i, c in enumerate(coords):
        border |= 0.5 * g.ext[i] * g.factor - np.abs(c) < g.ext[i] / g.T[i]
    inside = norm <= 1.0
    min_c = base_values[inside].min()
    alpha = base_values[~inside & border].max()
    beta = min(max_factor * alpha, min_c)
    f = lambda t: _sigmoid_ref(sig, 0.0, beta - alpha, beta - t, rec)  # noqa: E731
    offset = beta - quad(f, alpha, beta, epsabs=1e-14, epsrel=1e-12)[0]
    out = base_values.copy()
    for k in np.nonzero(~inside)[0]:
        x = base_values[k]
        if x < alpha:
            out[k] = offset
        elif x < beta:
            out[k] = quad(f, alpha, x, epsabs=1e-14, epsrel=1e-12)[0] + offset
    return out, alpha, beta


@pytest.mark.parametrize("case", [
    dict(kw=dict(dim=2, cells=(16, 12), covariance="exponential", corr_length=0.5, embedding_factor=3),
         sig="smoothstep", rec=1, mf=5.0),
    dict(kw=dict(dim=3, cells=(8, 6, 4), covariance="matern32", corr_length=0.3, embedding_factor=4),
         sig="smooth", rec=1, mf=5.0),
    dict(kw=dict(dim=2, cells=(12, 10), covariance="exponential", corr_length=(0.4, 0.1, -0.1, 0.3),
                 anisotropy="geometric", embedding_factor=4), sig="smoothstep", rec=3, mf=3.0),
    # factor 3 in 3D: the domain corner (radius sqrt 3) lies beyond the border (1.5), so
    # beta < alpha and every value below alpha becomes beta (the reference's arithmetic)
    dict(kw=dict(dim=3, cells=(8, 6, 4), covariance="matern32", corr_length=(0.3, 0.2, 0.25),
                 anisotropy="axiparallel", embedding_factor=3), sig="smooth", rec=1, mf=5.0, inverted=True),
])
def test_cofold_periodization_matches_restatement(oracle, case):
    """embedding.periodization = cofold: the oracle's C restatement against an independent
    numpy/scipy restatement over the classical fill (DCT matrix, and R2C with its padding)."""
    import pfb200
    base = pfb200.make_desc(**case["kw"])
    cof = pfb200.make_desc(**case["kw"], periodization="cofold", sigmoid=case["sig"],
                           cofold_recursions=case["rec"], cofold_max_factor=case["mf"])
    a = oracle.fill_matrix(base)
    b = oracle.fill_matrix(cof)
    want, alpha, beta = _cofold_numpy(oracle, cof, a, case["sig"], case["rec"], case["mf"])
    assert (alpha > beta) == case.get("inverted", False)
    assert np.abs(b - want).max() <= 1e-12 * np.abs(a).max()
    assert np.abs(a - b).max() > 1e-6 * np.abs(a).max()


def test_cofold_keeps_domain_values_and_lifts_the_rest(oracle):
    """Cofold never changes a value within the domain's extent (norm <= 1) and never lowers
    a value beyond it: values below the border maximum alpha are lifted to the offset."""
    import pfb200
    kw = dict(dim=2, cells=(16, 12), covariance="exponential", corr_length=0.5, embedding_factor=3)
    g = oracle.resolve(pfb200.make_desc(**kw))
    a = oracle.fill_matrix(pfb200.make_desc(**kw))
    b = oracle.fill_matrix(pfb200.make_desc(**kw, periodization="cofold"))
    j1, j0 = np.meshgrid(np.arange(g.T[1] // 2 + 1), np.arange(g.T[0] // 2 + 1), indexing="ij")
    norm = np.maximum(j0 * g.h[0] / g.ext[0], j1 * g.h[1] / g.ext[1]).ravel()
    inside = norm <= 1.0
    assert np.array_equal(a[inside], b[inside])
    assert (b[~inside] >= a[~inside]).all()


def test_cofold_rejects_negative_recursions(oracle):
    import pfb200
    d = pfb200.make_desc(dim=2, cells=(8, 8), periodization="cofold", cofold_recursions=-1)
    with pytest.raises(ValueError, match="cofoldRecursions"):
        oracle.resolve(d)
