"""Shared test helpers: descriptor construction and eigenvalue layout conversion."""
import numpy as np

import pfb200


def desc_of(cfg, **over):
    kw = dict(cfg)
    kw.update(over)
    dim = kw["dim"]
    cells = tuple(kw["cells"]) + (1,) * (3 - dim)
    kw["cells"] = cells
    return pfb200.make_desc(**{k: v for k, v in kw.items() if k in pfb200.make_desc.__code__.co_varnames})


def full_lambda(g, lam):
    """Eigenvalues in the reference storage layout -> full torus, numpy order."""
    dim = g.dim
    T = [g.T[i] for i in range(dim)]
    mb = g.matrix_backend
    if mb == pfb200.MATRIX_DCT:
        D = [t // 2 + 1 for t in T]
        Ds = [g.Ts[i] // 2 + 1 for i in range(dim)]
        L = lam.reshape(tuple(reversed(Ds)))
        if g.transposed:  # stored dims (0, d-1, d-2)
            L = np.swapaxes(L, 0, 1)
        idx = [np.minimum(np.arange(t), t - np.arange(t)) for t in reversed(T)]
        return L[np.ix_(*idx)]
    if mb == pfb200.MATRIX_R2C:
        T0c = T[0] // 2 + 1
        shp = [T0c] + [g.Ts[i] for i in range(1, dim)]
        L = lam.reshape(tuple(reversed(shp)))
        if g.transposed:
            L = np.swapaxes(L, 0, 1)
        full = np.zeros(tuple(reversed(T)))
        full[..., :T0c] = L
        # fill k0 > T0/2 by the point symmetry lambda(-k) = lambda(k)
        for k0 in range(T0c, T[0]):
            src = L[..., T[0] - k0]
            for ax in range(dim - 1):
                src = np.roll(np.flip(src, axis=ax), 1, axis=ax)
            full[..., k0] = src
        return full
    L = lam.reshape(tuple(reversed([g.Ts[i] for i in range(dim)])))
    if g.transposed:
        L = np.swapaxes(L, 0, 1)
    return L


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
