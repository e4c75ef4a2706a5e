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


# ---------------------------------------------------------------------------
# counter-based noise of the library, reproduced on the host
# ---------------------------------------------------------------------------
def _philox4x32_10(c, seed):
    """Philox4x32-10 (Salmon et al., SC 2011) on uint64 arrays holding 32-bit words."""
    m32 = np.uint64(0xFFFFFFFF)
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) & m32 for x in c)
    k0, k1 = np.uint64(seed & 0xFFFFFFFF), np.uint64((seed >> 32) & 0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        c0, c1, c2, c3 = ((p1 >> np.uint64(32)) ^ c1 ^ k0, p1 & m32, (p0 >> np.uint64(32)) ^ c3 ^ k1, p0 & m32)
        k0 = (k0 + np.uint64(0x9E3779B9)) & m32
        k1 = (k1 + np.uint64(0xBB67AE85)) & m32
    return c0, c1, c2, c3


def _box_muller(a, b, fp64):
    """u1 = (a + 1/2) 2^-32; u2 from all 32 bits of b (FP64 path) or its top 23 (FP32)."""
    u1 = (a.astype(np.float64) + 0.5) * 2.0 ** -32
    u2 = b.astype(np.float64) * 2.0 ** -32 if fp64 else (b >> np.uint64(9)).astype(np.float64) * 2.0 ** -23
    rad = np.sqrt(-2.0 * np.log(u1))
    ang = 2.0 * np.pi * u2 - np.pi
    return rad * np.cos(ang), rad * np.sin(ang)


def counter_noise(g, seed, fp64, epoch=0, chunk=1 << 21):
    """The device's seeded noise in the reference draw order (R2C field backend, even last
    extent): stored frequency s with last-axis index kl < T/2 takes words (x, y) of
    Philox(s, 0, 'pair', epoch); its partner kl + T/2 takes words (z, w) of the same call.
    Computed in slabs of about `chunk` pairs, so full-size tori fit in host memory."""
    dim = g.dim
    T = [g.T[i] for i in range(3)]
    T0c = T[0] // 2 + 1
    Tl = T[dim - 1]
    h = Tl // 2
    out = np.empty(int(g.noise))
    planes = T[1] if dim == 3 else 1
    per_plane = T0c * h
    step = max(1, chunk // per_plane)
    for p0 in range(0, planes, step):
        p1 = min(planes, p0 + step)
        if dim == 2:
            k0, kl = np.meshgrid(np.arange(T0c), np.arange(h), indexing="ij")
            k1 = np.zeros_like(k0)
        else:
            k0, k1, kl = np.meshgrid(np.arange(T0c), np.arange(p0, p1), np.arange(h), indexing="ij")

        def stored(kk):
            if dim == 2:
                return k0 + T0c * kk
            if g.transposed:
                return k0 + T0c * (kk + T[2] * k1)
            return k0 + T0c * (k1 + T[1] * kk)

        s0, s1 = stored(kl).ravel().astype(np.int64), stored(kl + h).ravel().astype(np.int64)
        x, y, z, w = _philox4x32_10((s0, np.zeros_like(s0), np.full_like(s0, 0x70616972),
                                     np.full_like(s0, epoch)), seed)
        out[2 * s0], out[2 * s0 + 1] = _box_muller(x, y, fp64)
        out[2 * s1], out[2 * s1 + 1] = _box_muller(z, w, fp64)
    return out
