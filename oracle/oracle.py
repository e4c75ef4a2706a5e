"""ctypes wrapper of oracle/liboracle.so, the FP64 CPU restatement of the
reference's circulant-embedding path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the product.  Parity with the reference
binary is unpinned (the reference cannot be built here and its tests hold no
golden vectors); the FFT conventions are pinned against scipy.fft.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "parafields-core_b200"))
import pfb200  # noqa: E402  (descriptor struct only; no CUDA library is loaded)

_lib = None


class Geom(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("n", C.c_int * 3), ("T", C.c_int * 3), ("Ts", C.c_int * 3),
        ("h", C.c_double * 3), ("ext", C.c_double * 3), ("factor", C.c_int),
        ("matrix_backend", C.c_int), ("field_backend", C.c_int), ("transposed", C.c_int),
        ("domain", C.c_uint64), ("N", C.c_uint64), ("Nc", C.c_uint64), ("D", C.c_uint64),
        ("spectrum", C.c_uint64), ("noise", C.c_uint64),
    ]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        D = C.POINTER(pfb200.FieldDesc)
        dp = C.POINTER(C.c_double)
        L.oc_resolve.argtypes = [D, C.POINTER(Geom), C.c_char_p, C.c_int]
        L.oc_covariance.argtypes = [D, dp]
        L.oc_covariance.restype = C.c_double
        L.oc_geometry.argtypes = [D, dp, dp]
        L.oc_fft.argtypes = [C.c_int, dp, C.c_int]
        L.oc_fft_axis.argtypes = [dp, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int]
        L.oc_r2c.argtypes = [C.c_int, C.POINTER(C.c_int), dp, dp]
        L.oc_c2r.argtypes = [C.c_int, C.POINTER(C.c_int), dp, dp]
        L.oc_dct1.argtypes = [C.c_int, C.POINTER(C.c_int), dp]
        L.oc_fill_matrix.argtypes = [D, dp, C.c_uint64]
        L.oc_spectrum.argtypes = [D, dp, C.POINTER(pfb200.EigStats)]
        L.oc_generate.argtypes = [D, dp, dp, dp, dp]
        L.oc_matvec.argtypes = [D, dp, C.c_int, dp, dp]
        L.oc_multiply_inverse.argtypes = [D, dp, dp, dp, C.POINTER(C.c_int)]
        L.oc_transform.argtypes = [C.c_int, C.c_double, dp, C.c_uint64]
        L.oc_num_threads.restype = C.c_int
        L.oc_set_num_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ints(v):
    return (C.c_int * len(v))(*[int(x) for x in v])


def set_threads(n):
    lib().oc_set_num_threads(int(n))


def num_threads():
    return lib().oc_num_threads()


def resolve(desc):
    g = Geom()
    err = C.create_string_buffer(256)
    st = lib().oc_resolve(C.byref(desc), C.byref(g), err, 256)
    if st:
        raise ValueError(err.value.decode())
    return g


def fft(x, sign):
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().oc_fft(a.size, _dp(a.view(np.float64)), sign)
    return a


def fft_axis(x, axis_param, sign):
    """x: numpy complex array with C-order shape (..., shape[1], shape[0]); axis in
    parafields numbering (0 = fastest)."""
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    shape = list(reversed(a.shape))
    lib().oc_fft_axis(_dp(a.view(np.float64)), len(shape), _ints(shape), axis_param, sign)
    return a


def r2c(x):
    """x: real array, C-order shape (T2, T1, T0) -> complex (T2, T1, T0//2+1)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    T = list(reversed(x.shape))
    out = np.empty(x.shape[:-1] + (T[0] // 2 + 1,), dtype=np.complex128)
    lib().oc_r2c(len(T), _ints(T), _dp(x), _dp(out.view(np.float64)))
    return out


def c2r(X, T0):
    X = np.ascontiguousarray(X, dtype=np.complex128)
    T = [T0] + list(reversed(X.shape[:-1]))
    out = np.empty(X.shape[:-1] + (T0,), dtype=np.float64)
    lib().oc_c2r(len(T), _ints(T), _dp(X.view(np.float64)), _dp(out))
    return out


def dct1(x):
    a = np.ascontiguousarray(x, dtype=np.float64).copy()
    m = list(reversed(a.shape))
    lib().oc_dct1(len(m), _ints(m), _dp(a))
    return a


def covariance(desc, x):
    """c at the already transformed distance vector x (covariance.hh:296-823)"""
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().oc_covariance(C.byref(desc), _dp(x))


def geometry(desc, x):
    """the anisotropy transform of a physical distance vector (covariance.hh:18-138)"""
    v = np.zeros(3)
    x = np.asarray(x, dtype=np.float64).ravel()
    v[: x.size] = x
    x = v
    out = np.zeros(3)
    lib().oc_geometry(C.byref(desc), _dp(np.ascontiguousarray(x)), _dp(out))
    return out


def prescribed_covariance(desc, lag):
    """c(h) of the configured covariance at the physical lag vector h"""
    return covariance(desc, geometry(desc, lag))


def fill_matrix(desc):
    g = resolve(desc)
    if g.matrix_backend == pfb200.MATRIX_DCT:
        cells = [g.T[i] // 2 + 1 if i < g.dim else 1 for i in range(3)]
    elif g.matrix_backend == pfb200.MATRIX_R2C:
        cells = [2 * (g.T[0] // 2 + 1)] + [g.T[i] if i < g.dim else 1 for i in (1, 2)]
    else:
        cells = [g.T[i] if i < g.dim else 1 for i in range(3)]
    out = np.empty(int(np.prod(cells)), dtype=np.float64)
    st = lib().oc_fill_matrix(C.byref(desc), _dp(out), out.size)
    assert st == 0, st
    return out


def spectrum(desc):
    """(lambda in the reference's storage layout, stats dict, status)."""
    g = resolve(desc)
    lam = np.empty(g.spectrum, dtype=np.float64)
    st = pfb200.EigStats()
    status = lib().oc_spectrum(C.byref(desc), _dp(lam), C.byref(st))
    return lam, st.as_dict(), status


def generate(desc, lam, noise):
    g = resolve(desc)
    assert noise.size == g.noise and noise.dtype == np.float64
    field = np.empty(g.domain, dtype=np.float64)
    spare = np.empty(g.domain, dtype=np.float64)
    st = lib().oc_generate(C.byref(desc), _dp(lam), _dp(np.ascontiguousarray(noise)), _dp(field),
                           _dp(spare))
    assert st == 0, st
    return field, spare


def matvec(desc, lam, op, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    st = lib().oc_matvec(C.byref(desc), _dp(lam), op, _dp(x), _dp(out))
    assert st == 0, st
    return out


def multiply_inverse(desc, lam, b):
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.empty_like(b)
    it = C.c_int()
    st = lib().oc_multiply_inverse(C.byref(desc), _dp(lam), _dp(b), _dp(x), C.byref(it))
    assert st == 0, st
    return x, it.value


def transform(kind, v, boxcox_lambda=0.0):
    a = np.ascontiguousarray(v, dtype=np.float64).copy()
    k = pfb200.TRANSFORMS[kind] if isinstance(kind, str) else int(kind)
    lib().oc_transform(k, boxcox_lambda, _dp(a), a.size)
    return a


def noise(seed, count):
    """Seeded N(0,1) doubles (numpy PCG64 + its standard normal method); the same
    buffer is fed to the oracle and to the GPU in the reference's draw order."""
    return np.random.default_rng(seed).standard_normal(int(count))


# ---------------------------------------------------------------------------
# learned boundary correction of the CG preconditioner: M = D P0 D (no counterpart in
# the reference; the library's kernels are in csrc/pf_learned.cuh).  FP64 restatement of
# its features, scaling, loss and gradient, used to check the device gradients.
# ---------------------------------------------------------------------------
def learned_features(desc):
    g = resolve(desc)
    dim = g.dim
    lens = []
    cl = list(desc.corr_length)
    for i in range(3):
        if i >= dim:
            lens.append(1.0)
        elif desc.anisotropy == 0:
            lens.append(cl[0])
        elif desc.anisotropy == 1:
            lens.append(cl[i])
        else:
            lens.append(float(np.sqrt(sum(cl[i * dim + j] ** 2 for j in range(dim)))))
    feats = []
    for a in range(3):
        n = g.n[a]
        m = np.arange(n)
        dist = np.minimum(m + 0.5, n - m - 0.5)
        feats.append(dist * g.h[a] / lens[a])
    return g, feats


def learned_psi(theta, H, t):
    t = np.asarray(t, dtype=np.float64)
    w1, b1, w2, b2 = theta[:H], theta[H:2 * H], theta[2 * H:3 * H], theta[3 * H]
    return np.tanh(np.outer(t, w1) + b1) @ w2 + b2


def learned_scale(desc, theta, H):
    g, feats = learned_features(desc)
    dim = g.dim
    psi = [learned_psi(theta, H, feats[a]) if a < dim else np.zeros(g.n[a]) for a in range(3)]
    s = psi[2][:, None, None] + psi[1][None, :, None] + psi[0][None, None, :]   # (x2, x1, x0)
    return np.exp(s).ravel()


def learned_loss_grad(desc, lam, theta, H, B, X, residual=False):
    """L = (1/K) sum ||D P0 D b - x||^2 / ||x||^2 (or ||A(D P0 D b - x)||^2 / ||b||^2 with
    residual=True) and dL/dtheta (P0 = torus inverse, A the restricted covariance)."""
    g, feats = learned_features(desc)
    dim = g.dim
    n = [g.n[0], g.n[1], g.n[2]]
    d = learned_scale(desc, theta, H)
    K = len(B)
    loss = 0.0
    gcell = np.zeros_like(d)
    for b, x in zip(B, X):
        v = matvec(desc, lam, 2, d * b)
        e = d * v - x
        if residual:
            f = matvec(desc, lam, 0, e)
            nn = float(b @ b)
            loss += float(f @ f) / nn / K
            e = matvec(desc, lam, 0, f)
        else:
            nn = float(x @ x)
            loss += float(e @ e) / nn / K
        w = matvec(desc, lam, 2, d * e)
        gcell += (2.0 / (nn * K)) * (e * v + b * w) * d
    gc = gcell.reshape(n[2], n[1], n[0])
    gprof = [gc.sum(axis=(0, 1)), gc.sum(axis=(0, 2)), gc.sum(axis=(1, 2))]
    w1, b1, w2 = theta[:H], theta[H:2 * H], theta[2 * H:3 * H]
    grad = np.zeros(3 * H + 1)
    for a in range(dim):
        t = feats[a]
        A = np.tanh(np.outer(t, w1) + b1)                      # (m, H)
        gp = gprof[a]
        grad[2 * H:3 * H] += gp @ A
        dA = (1.0 - A ** 2) * w2
        grad[:H] += (gp * t) @ dA
        grad[H:2 * H] += gp @ dA
        grad[3 * H] += gp.sum()
    return loss, grad


# ---------------------------------------------------------------------------
# DCT/DST field backend (opt-in in the reference), FP64 restatement in numpy/scipy:
# DCTDSTFieldBackend::setType / set / backwardTransform / extendedFieldToField
# (include/parafields/backends/dctdstfieldbackend.hh:149-165, 326-438, 631-771) driven by
# Matrix::generateField (include/parafields/matrix.hh:342-367).  scipy.fft.dct/dst of type 1
# without normalization are FFTW's REDFT00/RODFT00.  With fftw.transposed the draws follow
# the transposed cell order; the transforms and the field do not depend on the layout.
# ---------------------------------------------------------------------------
def dctdst_noise_size(desc):
    dim = desc.dim
    factor = 1 if desc.periodic else desc.embedding_factor
    D = int(np.prod([factor * desc.cells[i] // 2 + 1 for i in range(dim)]))
    return D << dim


def generate_dctdst(desc, lam, noise):
    """Field of the reference's DCT/DST backend for DCT eigenvalues `lam` (natural layout,
    dim 0 fastest) and draws `noise` (type-major, then DCT cell index, dim 0 fastest).
    The first type replaces the field (the documented intent; the reference's non-additive
    extraction also adds, dctdstfieldbackend.hh:923)."""
    import scipy.fft as sf
    dim = desc.dim
    factor = 1 if desc.periodic else desc.embedding_factor
    n = [desc.cells[i] for i in range(dim)]
    T = [factor * c for c in n]
    D = [t // 2 + 1 for t in T]
    shape = tuple(reversed(D))  # numpy order (d-1, ..., 0)
    sq = np.sqrt(np.maximum(np.asarray(lam, dtype=np.float64), 0.0)).reshape(shape)
    Dtot = int(np.prod(D))
    # draw order: the backend's local cells, dims d-1 and d-2 swapped when fftw.transposed
    # (default for dim > 1; dctdstfieldbackend.hh:855-871 with matrix.hh:349-360)
    transposed = dim > 1 and (desc.transposed < 0 or desc.transposed != 0)
    stored = list(D)
    if transposed:
        stored[dim - 1], stored[dim - 2] = stored[dim - 2], stored[dim - 1]
    field = np.zeros(tuple(reversed(n)))
    for t in range(1 << dim):
        odd = [(t >> i) & 1 for i in range(dim)]
        r = np.asarray(noise[t * Dtot:(t + 1) * Dtot], dtype=np.float64).reshape(tuple(reversed(stored)))
        if transposed:
            r = np.swapaxes(r, 0, 1)
        X = sq * r * 2.0 ** (-dim / 2.0)
        for i in range(dim):
            ax = dim - 1 - i
            idx = [slice(None)] * dim
            if odd[i]:
                for e in (0, D[i] - 1):  # odd axis on its border: zero
                    idx[ax] = e
                    X[tuple(idx)] = 0.0
            else:
                for e in (0, D[i] - 1):  # even axis on its border: factor sqrt(2)
                    idx[ax] = e
                    X[tuple(idx)] *= np.sqrt(2.0)
        for i in range(dim):
            ax = dim - 1 - i
            if odd[i]:
                inner = [slice(None)] * dim
                inner[ax] = slice(1, D[i] - 1)
                Y = np.zeros_like(X)
                Y[tuple(inner)] = sf.dst(X[tuple(inner)], type=1, axis=ax)
                X = Y
            else:
                X = sf.dct(X, type=1, axis=ax)
        field += X[tuple(slice(0, c) for c in reversed(n))]
    return field.ravel()
