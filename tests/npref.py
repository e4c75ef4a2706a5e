"""Second, independent restatement of the reference's circulant-embedding path in
numpy + scipy.fft, for small sizes.  It shares no code with oracle/pf_oracle.c; the
tests require both restatements to agree, and tests/golden/make_golden.py stores
their outputs as fixtures.

Arrays here are numpy arrays in C order with shape (n_{d-1}, ..., n_0), i.e. the
reference's dimension 0 is the last numpy axis.
"""
import math

import numpy as np
import scipy.fft as sf

COV = {
    "matern": 4,
    "exponential": 0, "gaussian": 1, "spherical": 2, "separableExponential": 3,
    "matern32": 5, "matern52": 6, "dampedOscillation": 7, "gammaExponential": 8,
    "cauchy": 9, "generalizedCauchy": 10, "cubic": 11, "whiteNoise": 12,
}


def geometry(cfg, x):
    """covariance.hh:18-138; x has shape (..., dim) in parafields order."""
    dim = cfg["dim"]
    cl = np.atleast_1d(np.asarray(cfg["corr_length"], dtype=float))
    aniso = cfg.get("anisotropy", "none")
    if aniso == "none":
        return x * (1.0 / cl[0])
    if aniso == "axiparallel":
        return x * (1.0 / cl[:dim])
    A = cl[: dim * dim].reshape(dim, dim)
    return x @ np.linalg.inv(A).T


def covariance(cfg, xt):
    dim = cfg["dim"]
    var = cfg.get("variance", 1.0)
    c = cfg["covariance"]
    h = np.sqrt((xt ** 2).sum(axis=-1))
    if c == "exponential":
        return var * np.exp(-h)
    if c == "gaussian":
        return var * np.exp(-h * h)
    if c == "spherical":
        hh = np.minimum(h, 1.0)
        if dim == 3:
            v = 1 - 1.5 * hh + 0.5 * hh ** 3
        elif dim == 2:
            v = 1 - 2 / math.pi * (hh * np.sqrt(1 - hh ** 2) + np.arcsin(hh))
        else:
            v = 1 - hh
        return np.where(h > 1, 0.0, var * v)
    if c == "separableExponential":
        return var * np.exp(-np.abs(xt).sum(axis=-1))
    if c == "matern32":
        return var * (1 + math.sqrt(3) * h) * np.exp(-math.sqrt(3) * h)
    if c == "matern52":
        return var * (1 + math.sqrt(5) * h + 5 / 3 * h * h) * np.exp(-math.sqrt(5) * h)
    if c == "dampedOscillation":
        return var * np.exp(-h) * np.cos(h / math.sqrt(3) if dim == 3 else h)
    if c == "gammaExponential":
        return var * np.exp(-h ** cfg["exp_gamma"])
    if c == "cauchy":
        return var * (1 + h ** 2) ** -3.0
    if c == "generalizedCauchy":
        return var * (1 + h ** cfg["cauchy_alpha"]) ** (-cfg["cauchy_beta"])
    if c == "cubic":
        hh = np.minimum(h, 1.0)
        v = 1 - 7 * hh ** 2 + 8.75 * hh ** 3 - 3.5 * hh ** 5 + 0.75 * hh ** 7
        return np.where(h > 1, 0.0, var * v)
    if c == "matern":
        from scipy.special import gamma, kv
        nu = cfg["matern_nu"]
        z = np.sqrt(2 * nu) * h
        with np.errstate(invalid="ignore"):
            v = var * 2 ** (1 - nu) / gamma(nu) * z ** nu * kv(nu, np.where(z > 0, z, 1.0))
        return np.where(h < 1e-10, var, v)
    if c == "whiteNoise":
        return np.where((np.abs(xt) > 1e-10).any(axis=-1), 0.0, var)
    raise ValueError(c)


def torus(cfg):
    """Covariance on the whole torus with the classical mirroring (matrix.hh:615-638)."""
    dim = cfg["dim"]
    n = cfg["cells"][:dim]
    ext = cfg.get("extensions", [1.0] * dim)
    f = cfg.get("embedding_factor", 2)
    T = [f * c for c in n]
    axes = []
    for i in range(dim):
        h = ext[i] / n[i]
        c = np.arange(T[i]) * h
        c = np.where(c > 0.5 * ext[i] * f, c - ext[i] * f, c)
        axes.append(c)
    grids = np.meshgrid(*axes, indexing="ij")  # parafields order
    x = np.stack(grids, axis=-1)
    cov = covariance(cfg, geometry(cfg, x))
    return np.transpose(cov)  # numpy order (T_{d-1}, ..., T_0)


def spectrum_full(cfg):
    """Eigenvalues on the full torus, lambda = DFT(c)/N (real part)."""
    c = torus(cfg)
    return np.real(sf.fftn(c)) / c.size


def generate_r2c(cfg, lam_full, noise, transposed):
    """R2CFieldBackend generation (r2cfieldbackend.hh:305-325, matrix.hh:375-409):
    noise pair i belongs to stored complex entry i; 3D 'transposed' storage swaps the
    last two parafields dimensions."""
    dim = cfg["dim"]
    n = cfg["cells"][:dim]
    f = cfg.get("embedding_factor", 2)
    T = [f * c for c in n]
    T0c = T[0] // 2 + 1
    half_shape = tuple(reversed([T0c] + T[1:]))  # numpy order
    r1 = noise[0::2]
    r2 = noise[1::2]
    if transposed and dim == 3:
        # stored order: k0 fastest, then k2, then k1 -> numpy shape (T1, T2, T0c)
        r1 = r1.reshape(T[1], T[2], T0c).transpose(1, 0, 2)
        r2 = r2.reshape(T[1], T[2], T0c).transpose(1, 0, 2)
    else:
        r1 = r1.reshape(half_shape)
        r2 = r2.reshape(half_shape)
    lam = lam_full[..., :T0c]
    s = np.sqrt(lam)
    ks = np.meshgrid(*[np.arange(c) for c in reversed([T0c] + T[1:])], indexing="ij")
    selfc = np.ones(half_shape, dtype=bool)
    for ax, k in enumerate(ks):
        Ti = list(reversed(T))[ax]
        selfc &= (2 * k) % Ti == 0
    X = np.where(selfc, s * r1 + 0j, (s / math.sqrt(2)) * r1 + 1j * (s / math.sqrt(2)) * r2)
    out = sf.irfftn(X, s=tuple(reversed(T))) * np.prod(T)
    sl = tuple(slice(0, c) for c in reversed(n))
    return out[sl]


def matvec(cfg, lam_full, x, op):
    """multiplyExtended / Root / InverseExtended (matrix.hh:1443-1646): embed, R2C/N,
    multiply, C2R, restrict."""
    dim = cfg["dim"]
    n = cfg["cells"][:dim]
    f = cfg.get("embedding_factor", 2)
    T = [f * c for c in n]
    N = np.prod(T)
    tor = np.zeros(tuple(reversed(T)))
    tor[tuple(slice(0, c) for c in reversed(n))] = x
    X = sf.rfftn(tor) / N
    lam = lam_full[..., : T[0] // 2 + 1]
    fac = {0: lam, 1: np.sqrt(lam), 2: 1.0 / lam}[op]
    y = sf.irfftn(X * fac, s=tuple(reversed(T))) * N
    return y[tuple(slice(0, c) for c in reversed(n))]
