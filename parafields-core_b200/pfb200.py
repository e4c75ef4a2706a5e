"""ctypes binding of libpfcuda.so, the C ABI in include/parafields_b200.h.

This is the Python-side mirror of the reference's Matrix API for the
circulant-embedding path (include/parafields/matrix.hh:142-421, 1443-1646) used
by the tests and the benchmark.  The CUDA library is loaded on first use and the
binding raises if it is missing: there is no CPU fallback.

Array arguments are numpy arrays (host memory) or torch CUDA tensors (device
memory, passed by data_ptr()).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PFB200_LIB", os.path.join(HERE, "lib", "libpfcuda.so"))

# --- enums (include/parafields_b200.h) ---------------------------------------
PF_OK, PF_ERR_NEG_EIGEN, PF_ERR_CONFIG, PF_ERR_OOM, PF_ERR_CUDA = 0, 1, 2, 3, 4
PF_ERR_NOT_CONVERGED, PF_ERR_TIMEOUT, PF_ERR_STATE, PF_ERR_ARG, PF_ERR_IO = 5, 6, 7, 8, 9

COVARIANCES = {
    "exponential": 0, "gaussian": 1, "spherical": 2, "separableExponential": 3,
    "matern": 4, "matern32": 5, "matern52": 6, "dampedOscillation": 7,
    "gammaExponential": 8, "cauchy": 9, "generalizedCauchy": 10, "cubic": 11,
    "whiteNoise": 12,
    # the caller supplies the matrix cells (Plan.spectrum_build_values)
    "custom-iso": 13, "custom-aniso": 13,
}
ANISOTROPIES = {"none": 0, "axiparallel": 1, "geometric": 2}
TRANSFORMS = {"none": 0, "logNormal": 1, "foldedNormal": 2, "sign": 3, "boxCox": 4}
PERIODIZATIONS = {"classical": 0, "merge": 1, "fold": 2, "cofold": 3}
SIGMOIDS = {"smoothstep": 0, "smooth": 1}
COMBINES = {"radialPlus": 0, "radial": 1, "tensor": 2}
MATRIX_DCT, MATRIX_R2C, MATRIX_DFT = 0, 1, 2
FIELD_R2C, FIELD_DFT, FIELD_DCTDST = 0, 1, 2
PREC_F64, PREC_F32 = 0, 1
EIGCHECK_CORRECTED, EIGCHECK_REFERENCE = 0, 1
OP_MUL, OP_ROOT, OP_INVEXT = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
CG_REFERENCE, CG_RESIDUAL = 0, 1


class FieldDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("cells", C.c_int32 * 3), ("extensions", C.c_double * 3),
        ("embedding_factor", C.c_int32), ("periodic", C.c_int32), ("covariance", C.c_int32),
        ("variance", C.c_double), ("anisotropy", C.c_int32), ("corr_length", C.c_double * 9),
        ("matern_nu", C.c_double), ("exp_gamma", C.c_double), ("cauchy_alpha", C.c_double),
        ("cauchy_beta", C.c_double), ("approximate", C.c_int32), ("threshold", C.c_double),
        ("transposed", C.c_int32), ("matrix_backend", C.c_int32), ("field_backend", C.c_int32),
        ("precision", C.c_int32), ("eigen_check", C.c_int32), ("cg_iterations", C.c_int32),
        ("transform", C.c_int32), ("boxcox_lambda", C.c_double),
        ("periodization", C.c_int32), ("sigmoid", C.c_int32), ("sigmoid_combine", C.c_int32),
        ("merge_recursions", C.c_int32), ("sigmoid_start", C.c_double), ("sigmoid_end", C.c_double),
        ("fold_max_factor", C.c_double), ("fold_recursions", C.c_int32), ("cofold_recursions", C.c_int32),
        ("cofold_max_factor", C.c_double),
    ]


class EigStats(C.Structure):
    _fields_ = [("small", C.c_uint32), ("zero", C.c_uint32), ("negative", C.c_uint32),
                ("pad_", C.c_uint32), ("smallest", C.c_double)]

    def as_dict(self):
        return {"small": self.small, "zero": self.zero, "negative": self.negative,
                "smallest": self.smallest}


class PlanInfo(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("cells", C.c_int32 * 3), ("ext_cells", C.c_int32 * 3),
        ("matrix_backend", C.c_int32), ("field_backend", C.c_int32), ("transposed", C.c_int32),
        ("precision", C.c_int32), ("domain_size", C.c_uint64), ("ext_size", C.c_uint64),
        ("spectrum_size", C.c_uint64), ("noise_size", C.c_uint64), ("device_bytes", C.c_uint64),
    ]


class CgOpts(C.Structure):
    _fields_ = [("mode", C.c_int32), ("max_iterations", C.c_int32), ("tolerance", C.c_double),
                ("inner_fp32", C.c_int32), ("precondition", C.c_int32)]


class CgReport(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("refinements", C.c_int32),
                ("relative_residual", C.c_double)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_uint64), ("total_ms", C.c_double),
                ("bytes", C.c_double)]


def make_desc(dim=2, cells=(16, 16), extensions=None, covariance="exponential", variance=1.0,
              corr_length=0.05, anisotropy=None, embedding_factor=2, periodic=False,
              approximate=False, threshold=1e-14, transposed=-1, matrix_backend=-1,
              field_backend=-1, precision=PREC_F64, eigen_check=EIGCHECK_CORRECTED,
              cg_iterations=100, transform="none", boxcox_lambda=0.0, matern_nu=0.5,
              exp_gamma=1.0, cauchy_alpha=1.0, cauchy_beta=1.0, periodization="classical",
              sigmoid="smoothstep", sigmoid_combine="radialPlus", merge_recursions=99,
              sigmoid_start=1.0, sigmoid_end=-1.0, fold_max_factor=1.0, fold_recursions=99,
              cofold_max_factor=5.0, cofold_recursions=1) -> FieldDesc:
    """Builds a descriptor from values named after the reference's config keys."""
    d = FieldDesc()
    d.dim = dim
    for i in range(3):
        d.cells[i] = int(cells[i]) if i < dim else 1
        d.extensions[i] = float(extensions[i]) if (extensions is not None and i < dim) else 1.0
    d.embedding_factor = embedding_factor
    d.periodic = int(bool(periodic))
    d.covariance = COVARIANCES[covariance] if isinstance(covariance, str) else int(covariance)
    d.variance = variance
    cl = np.atleast_1d(np.asarray(corr_length, dtype=np.float64)).ravel()
    if anisotropy is None:
        if cl.size == 1:
            anisotropy = "none"
        elif cl.size == dim:
            anisotropy = "axiparallel"
        elif cl.size == dim * dim:
            anisotropy = "geometric"
        else:
            raise ValueError("stochastic.corrLength needs 1, dim or dim*dim values")
    d.anisotropy = ANISOTROPIES[anisotropy] if isinstance(anisotropy, str) else int(anisotropy)
    for i in range(9):
        d.corr_length[i] = float(cl[i]) if i < cl.size else 0.0
    d.matern_nu, d.exp_gamma = matern_nu, exp_gamma
    d.cauchy_alpha, d.cauchy_beta = cauchy_alpha, cauchy_beta
    d.approximate = int(bool(approximate))
    d.threshold = threshold
    d.transposed = transposed
    d.matrix_backend = matrix_backend
    d.field_backend = field_backend
    d.precision = precision
    d.eigen_check = eigen_check
    d.cg_iterations = cg_iterations
    d.transform = TRANSFORMS[transform] if isinstance(transform, str) else int(transform)
    d.boxcox_lambda = boxcox_lambda
    d.periodization = PERIODIZATIONS[periodization] if isinstance(periodization, str) else int(periodization)
    d.sigmoid = SIGMOIDS[sigmoid] if isinstance(sigmoid, str) else int(sigmoid)
    d.sigmoid_combine = COMBINES[sigmoid_combine] if isinstance(sigmoid_combine, str) else int(sigmoid_combine)
    d.merge_recursions = merge_recursions
    d.sigmoid_start, d.sigmoid_end = sigmoid_start, sigmoid_end
    d.fold_max_factor, d.fold_recursions = fold_max_factor, fold_recursions
    d.cofold_max_factor, d.cofold_recursions = cofold_max_factor, cofold_recursions
    return d


_lib = None


class Peaks(C.Structure):
    _fields_ = [("fp32_ffma_tflops", C.c_double), ("fp32_ffma2_tflops", C.c_double),
                ("fp64_dfma_tflops", C.c_double), ("sm_clock_mhz", C.c_double), ("sms", C.c_int32),
                ("pad_", C.c_int32)]


def lib():
    """Loads libpfcuda.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libpfcuda.so not built ({LIB_PATH}); run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    vp, u64, i32 = C.c_void_p, C.c_uint64, C.c_int32
    sig = {
        "pf_field_desc_init": (None, [C.POINTER(FieldDesc)]),
        "pf_plan_create": (i32, [C.POINTER(FieldDesc), C.POINTER(vp)]),
        "pf_plan_destroy": (None, [vp]),
        "pf_plan_set_stream": (i32, [vp, vp]),
        "pf_plan_get_info": (i32, [vp, C.POINTER(PlanInfo)]),
        "pf_spectrum_build": (i32, [vp, C.POINTER(EigStats)]),
        "pf_spectrum_copy": (i32, [vp, vp, u64]),
        "pf_spectrum_build_values": (i32, [vp, vp, u64, i32, C.POINTER(EigStats)]),
        "pf_generate": (i32, [vp, vp, i32, u64, vp, i32, i32]),
        "pf_generate_batch": (i32, [vp, u64, i32, vp, i32, i32]),
        "pf_export_noise": (i32, [vp, u64, C.c_uint32, vp, i32]),
        "pf_matvec": (i32, [vp, i32, i32, vp, vp, i32]),
        "pf_matvec_static": (i32, [vp, i32, vp, vp]),
        "pf_multiply_inverse": (i32, [vp, vp, vp, i32, C.POINTER(CgOpts), C.POINTER(CgReport)]),
        "pf_multiply_inverse_batch": (i32, [vp, vp, vp, i32, i32, C.POINTER(CgOpts), C.POINTER(CgReport), i32]),
        "pf_apply_transform": (i32, [vp, i32, vp, u64, i32]),
        "pf_profile_enable": (i32, [vp, i32]),
        "pf_profile_read": (i32, [vp, C.POINTER(KernelTime), i32, C.POINTER(i32)]),
        "pf_launch_count": (u64, [vp]),
        "pf_ensemble_create": (i32, [C.POINTER(FieldDesc), i32, u64, C.POINTER(vp)]),
        "pf_ensemble_destroy": (None, [vp]),
        "pf_ensemble_info": (i32, [vp, C.POINTER(i32), C.POINTER(u64), C.POINTER(u64)]),
        "pf_ensemble_spectra": (i32, [vp, C.POINTER(EigStats), C.POINTER(i32)]),
        "pf_ensemble_generate": (i32, [vp, vp, i32]),
        "pf_ensemble_launch": (i32, [vp, vp]),
        "pf_ensemble_autotune": (i32, [vp, i32, C.POINTER(i32)]),
        "pf_ensemble_device_output": (vp, [vp]),
        "pf_ensemble_launches_per_replay": (u64, [vp]),
        "pf_learned_create": (i32, [vp, i32, u64, C.POINTER(vp)]),
        "pf_learned_destroy": (None, [vp]),
        "pf_learned_param_count": (i32, [vp]),
        "pf_learned_get_params": (i32, [vp, vp]),
        "pf_learned_set_params": (i32, [vp, vp]),
        "pf_learned_loss_grad": (i32, [vp, vp, vp, i32, i32, i32, C.POINTER(C.c_double), vp]),
        "pf_learned_train": (i32, [vp, vp, vp, i32, i32, i32, C.c_double, i32, C.POINTER(C.c_double)]),
        "pf_learned_apply": (i32, [vp, vp, vp, i32]),
        "pf_plan_set_preconditioner": (i32, [vp, vp]),
        "pf_learned_set_loss": (i32, [vp, i32]),
        "pf_plan_autotune": (i32, [vp, i32, C.POINTER(i32)]),
        "pf_wisdom_export": (i32, [C.c_char_p, u64, C.POINTER(u64)]),
        "pf_wisdom_import": (i32, [C.c_char_p]),
        "pf_wisdom_forget": (None, []),
        "pf_measure_peaks": (i32, [i32, C.POINTER(Peaks)]),
        "pf_field_write": (i32, [C.c_char_p, i32, C.POINTER(i32), C.POINTER(C.c_double), vp, i32, i32]),
        "pf_field_read": (i32, [C.c_char_p, i32, C.POINTER(i32), vp, i32, i32]),
        "pf_last_error_string": (C.c_char_p, []),
        "pf_version": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class PfError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[pf status {status}] {msg}")
        self.status = status


class NegativeEigenvalueError(PfError):
    """Mirror of parafields::NegativeEigenvalueError (exceptions.hh:8-15)."""


def _check(st):
    if st != PF_OK:
        msg = lib().pf_last_error_string().decode()
        if st == PF_ERR_NEG_EIGEN:
            raise NegativeEigenvalueError(st, msg)
        raise PfError(st, msg)


def _numel(a):
    return a.size if isinstance(a, np.ndarray) else a.numel()


def _itemsize(a):
    return a.itemsize if isinstance(a, np.ndarray) else a.element_size()


def _need(a, count, itemsize, what):
    """the library writes/reads raw pointers: refuse buffers smaller than the call needs"""
    if a is None:
        return
    if _numel(a) < count or _itemsize(a) != itemsize:
        raise ValueError(f"{what}: buffer of {_numel(a)} x {_itemsize(a)} bytes, "
                         f"the call needs {count} x {itemsize} bytes")


def _ptr(a):
    """(pointer, memory kind) for a numpy array or a torch CUDA tensor."""
    if a is None:
        return None, MEM_HOST
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data, MEM_HOST
    # torch tensor
    assert a.is_contiguous()
    return a.data_ptr(), (MEM_DEVICE if a.is_cuda else MEM_HOST)


class Plan:
    """One field configuration on the GPU (the reference's Matrix object)."""

    def __init__(self, desc: FieldDesc):
        self.desc = desc
        h = C.c_void_p()
        _check(lib().pf_plan_create(C.byref(desc), C.byref(h)))
        self.h = h
        self.info = PlanInfo()
        _check(lib().pf_plan_get_info(self.h, C.byref(self.info)))

    def close(self):
        if self.h:
            lib().pf_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def domain_shape(self):
        """numpy shape of a field (dimension 0 fastest => reversed)."""
        return tuple(self.info.cells[i] for i in reversed(range(self.info.dim)))

    def set_stream(self, stream_handle: int):
        _check(lib().pf_plan_set_stream(self.h, C.c_void_p(stream_handle)))

    def spectrum_build(self):
        st = EigStats()
        _check(lib().pf_spectrum_build(self.h, C.byref(st)))
        return st.as_dict()

    def spectrum_build_values(self, values):
        """fillTransformedMatrix with caller-computed covariance values on the matrix cells
        (numpy float64 or a torch CUDA float64 tensor)."""
        if isinstance(values, np.ndarray):
            values = np.ascontiguousarray(values, dtype=np.float64)
        ptr, mem = _ptr(values)
        st = EigStats()
        n = values.size if isinstance(values, np.ndarray) else values.numel()
        _check(lib().pf_spectrum_build_values(self.h, ptr, n, mem, C.byref(st)))
        return st.as_dict()

    def spectrum(self):
        out = np.empty(self.info.spectrum_size, dtype=np.float64)
        _check(lib().pf_spectrum_copy(self.h, out.ctypes.data, out.size))
        return out

    def _field_dtype(self, precision=None):
        p = self.info.precision if precision is None else precision
        return np.float64 if p == PREC_F64 else np.float32

    def _fsize(self):
        return 8 if self.info.precision == PREC_F64 else 4

    def generate(self, noise=None, seed=0, out=None, apply_transform=False):
        if out is None:
            out = np.empty(self.info.domain_size, dtype=self._field_dtype())
        _need(out, self.info.domain_size, self._fsize(), "generate out")
        _need(noise, self.info.noise_size, 8, "generate noise")
        nptr, nmem = _ptr(noise)
        optr, omem = _ptr(out)
        _check(lib().pf_generate(self.h, nptr, nmem, seed, optr, omem, int(apply_transform)))
        return out

    def export_noise(self, seed, epoch=0, out=None):
        """the noise of a seeded realization in the reference's draw order (doubles)"""
        if out is None:
            out = np.empty(self.info.noise_size, dtype=np.float64)
        _need(out, self.info.noise_size, 8, "export_noise out")
        ptr, mem = _ptr(out)
        _check(lib().pf_export_noise(self.h, seed, epoch, ptr, mem))
        return out

    def generate_batch(self, seed, count, out=None, apply_transform=False):
        if out is None:
            out = np.empty(self.info.domain_size * count, dtype=self._field_dtype())
        _need(out, self.info.domain_size * count, self._fsize(), "generate_batch out")
        optr, omem = _ptr(out)
        _check(lib().pf_generate_batch(self.h, seed, count, optr, omem, int(apply_transform)))
        return out

    def matvec(self, x, op=OP_MUL, precision=PREC_F64, out=None):
        if out is None:
            out = np.empty_like(x)
        es = 8 if precision == PREC_F64 else 4
        _need(x, self.info.domain_size, es, "matvec in")
        _need(out, self.info.domain_size, es, "matvec out")
        iptr, mem = _ptr(x)
        optr, _ = _ptr(out)
        _check(lib().pf_matvec(self.h, op, precision, iptr, optr, mem))
        return out

    def multiply_inverse(self, b, x=None, mode=CG_REFERENCE, tolerance=1e-8, max_iterations=0,
                         inner_fp32=False, precondition=True):
        if x is None:
            x = np.empty_like(b)
        _need(b, self.info.domain_size, 8, "multiply_inverse b")
        _need(x, self.info.domain_size, 8, "multiply_inverse x")
        opts = CgOpts(mode, max_iterations, tolerance, int(inner_fp32), int(precondition))
        rep = CgReport()
        bptr, mem = _ptr(b)
        xptr, _ = _ptr(x)
        _check(lib().pf_multiply_inverse(self.h, bptr, xptr, mem, C.byref(opts), C.byref(rep)))
        return x, {"iterations": rep.iterations, "refinements": rep.refinements,
                   "relative_residual": rep.relative_residual}

    def multiply_inverse_batch(self, B, X=None, lanes=2, mode=CG_REFERENCE, tolerance=1e-8, max_iterations=0,
                               inner_fp32=False, precondition=True):
        """count right-hand sides (rows of B, prod(cells) doubles each) solved with up to
        `lanes` solves in flight; returns (X, list of reports)"""
        if X is None:
            X = np.empty_like(B)
        count = B.shape[0]
        _need(B, self.info.domain_size * count, 8, "multiply_inverse_batch B")
        _need(X, self.info.domain_size * count, 8, "multiply_inverse_batch X")
        opts = CgOpts(mode, max_iterations, tolerance, int(inner_fp32), int(precondition))
        reps = (CgReport * count)()
        bptr, mem = _ptr(B)
        xptr, _ = _ptr(X)
        _check(lib().pf_multiply_inverse_batch(self.h, bptr, xptr, count, mem, C.byref(opts), reps, lanes))
        return X, [{"iterations": r.iterations, "refinements": r.refinements,
                    "relative_residual": r.relative_residual} for r in reps]

    def apply_transform(self, data, precision=PREC_F64):
        ptr, mem = _ptr(data)
        n = data.size if isinstance(data, np.ndarray) else data.numel()
        _check(lib().pf_apply_transform(self.h, precision, ptr, n, mem))
        return data

    def profile(self, enable=True):
        _check(lib().pf_profile_enable(self.h, int(enable)))

    def profile_read(self):
        cap = 64
        arr = (KernelTime * cap)()
        n = C.c_int32()
        _check(lib().pf_profile_read(self.h, arr, cap, C.byref(n)))
        return [{"name": arr[i].name.decode(), "launches": arr[i].launches,
                 "total_ms": arr[i].total_ms, "bytes": arr[i].bytes} for i in range(n.value)]

    def autotune(self, repetitions=3):
        """Measured planning of the realization passes; True if it timed candidates (False
        when every pass came from the wisdom table)."""
        t = C.c_int32()
        _check(lib().pf_plan_autotune(self.h, repetitions, C.byref(t)))
        return bool(t.value)

    def launch_count(self):
        return int(lib().pf_launch_count(self.h))


class Ensemble:
    """Many independent fields (own sizes and covariances) generated together: one FP64
    spectrum per field, all realization passes replayed from one captured CUDA graph."""

    def __init__(self, descs, seed=0):
        arr = (FieldDesc * len(descs))(*descs)
        h = C.c_void_p()
        _check(lib().pf_ensemble_create(arr, len(descs), seed, C.byref(h)))
        self.h = h
        self.count = len(descs)
        self.precision = descs[0].precision
        n = C.c_int32()
        tot = C.c_uint64()
        offs = (C.c_uint64 * (self.count + 1))()
        _check(lib().pf_ensemble_info(self.h, C.byref(n), C.byref(tot), offs))
        self.total = int(tot.value)
        self.offsets = np.array(offs[:], dtype=np.int64)

    def spectra(self):
        stats = (EigStats * self.count)()
        failed = C.c_int32()
        _check(lib().pf_ensemble_spectra(self.h, stats, C.byref(failed)))
        return [s.as_dict() for s in stats]

    def generate(self, out=None):
        if out is None:
            out = np.empty(self.total, dtype=np.float64 if self.precision == PREC_F64 else np.float32)
        ptr, mem = _ptr(out)
        _check(lib().pf_ensemble_generate(self.h, ptr, mem))
        return out

    def autotune(self, repetitions=1):
        """measured planning of every field; returns the number of fields timed"""
        t = C.c_int32()
        _check(lib().pf_ensemble_autotune(self.h, repetitions, C.byref(t)))
        return t.value

    def launch(self, stream=None):
        _check(lib().pf_ensemble_launch(self.h, stream))

    def launches_per_replay(self):
        return int(lib().pf_ensemble_launches_per_replay(self.h))

    def field(self, flat, i):
        return flat[self.offsets[i]:self.offsets[i + 1]]

    def close(self):
        if self.h:
            lib().pf_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Learned:
    """Learned boundary correction M = D P0 D of a plan's CG preconditioner."""

    def __init__(self, plan, hidden=8, seed=0, residual_loss=False):
        h = C.c_void_p()
        _check(lib().pf_learned_create(plan.h, hidden, seed, C.byref(h)))
        self.h = h
        _check(lib().pf_learned_set_loss(self.h, int(residual_loss)))
        self.plan = plan
        self.hidden = hidden
        self.n = int(lib().pf_learned_param_count(self.h))

    @property
    def params(self):
        out = np.empty(self.n)
        _check(lib().pf_learned_get_params(self.h, out.ctypes.data))
        return out

    @params.setter
    def params(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        _check(lib().pf_learned_set_params(self.h, v.ctypes.data))

    def loss_grad(self, B, X, fp32=False):
        bptr, mem = _ptr(B)
        xptr, _ = _ptr(X)
        count = B.shape[0]
        loss = C.c_double()
        grad = np.empty(self.n)
        _check(lib().pf_learned_loss_grad(self.h, bptr, xptr, count, mem, int(fp32), C.byref(loss),
                                          grad.ctypes.data))
        return loss.value, grad

    def train(self, B, X, epochs, lr=0.02, fp32=True):
        bptr, mem = _ptr(B)
        xptr, _ = _ptr(X)
        loss = C.c_double()
        _check(lib().pf_learned_train(self.h, bptr, xptr, B.shape[0], mem, epochs, lr, int(fp32), C.byref(loss)))
        return loss.value

    def apply(self, r, out=None):
        if out is None:
            out = np.empty_like(r)
        rptr, mem = _ptr(r)
        optr, _ = _ptr(out)
        _check(lib().pf_learned_apply(self.h, rptr, optr, mem))
        return out

    def attach(self, enable=True):
        _check(lib().pf_plan_set_preconditioner(self.plan.h, self.h if enable else None))

    def close(self):
        if self.h:
            lib().pf_learned_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def wisdom_export():
    need = C.c_uint64()
    _check(lib().pf_wisdom_export(None, 0, C.byref(need)))
    buf = C.create_string_buffer(int(need.value))
    _check(lib().pf_wisdom_export(buf, need.value, C.byref(need)))
    return buf.value.decode()


def wisdom_import(text):
    _check(lib().pf_wisdom_import(text.encode()))


def wisdom_forget():
    lib().pf_wisdom_forget()


def measure_peaks(device=0):
    """CUDA-core FP32 (FFMA, FFMA2) and FP64 (DFMA) throughput of `device` in TFLOP/s."""
    p = Peaks()
    _check(lib().pf_measure_peaks(device, C.byref(p)))
    return {"fp32_ffma_tflops": p.fp32_ffma_tflops, "fp32_ffma2_tflops": p.fp32_ffma2_tflops,
            "fp64_dfma_tflops": p.fp64_dfma_tflops, "sm_clock_mhz": p.sm_clock_mhz, "sms": p.sms}


def write_field(base, data, cells, extensions):
    """writeToFile's stochastic part: `data` (numpy array or CUDA tensor, float64 or float32,
    dimension 0 fastest) to <base>.stoch.h5 (dataset /stochastic, F64LE) and <base>.xdmf."""
    dim = len(cells)
    ptr, mem = _ptr(data)
    prec = PREC_F64 if str(getattr(data, "dtype", "")).endswith("float64") else PREC_F32
    _check(lib().pf_field_write(str(base).encode(), dim, (C.c_int32 * dim)(*cells),
                                (C.c_double * dim)(*extensions), ptr, prec, mem))


def read_field(base, cells, out=None, precision=PREC_F64):
    """StochasticPart(traits, fileName): <base>.stoch.h5 into `out` (numpy array or CUDA
    tensor; a new float64 / float32 numpy array when None)."""
    dim = len(cells)
    n = int(np.prod(cells))
    if out is None:
        out = np.empty(n, dtype=np.float64 if precision == PREC_F64 else np.float32)
    else:
        precision = PREC_F64 if str(getattr(out, "dtype", "")).endswith("float64") else PREC_F32
    ptr, mem = _ptr(out)
    _check(lib().pf_field_read(str(base).encode(), dim, (C.c_int32 * dim)(*cells), ptr, precision, mem))
    return out
