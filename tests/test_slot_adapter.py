"""parafields_b200::GpuMatrix<Traits> (parafields-core_b200/include/parafields_b200/gpumatrix.hh)
in the reference's IsoMatrix/AnisoMatrix template slot (randomfield.hh:42-47).

CPU: the adapter compiles and links inside a RandomField stand-in that declares the
reference's member names, friend declarations and call forms (tests/cpp/slot_main.cc).
GPU: through that stand-in, generate(seed) with the reference's CppRNGBackend stream,
timesMatrix, timesMatrixRoot, timesInverseMatrix and generate after refineMatrix agree
with the oracle (or with the library's own CG) on the same noise; a user covariance
functor passed to fillMatrix (custom-iso) gives the field of the equal built-in
covariance."""
import os
import subprocess

import numpy as np
import pytest

import pfb200
from helpers import desc_of, rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CFG2 = """
[grid]
cells = 48 40
extensions = 1 1
[stochastic]
variance = 1.3
covariance = {cov}
anisotropy = {aniso}
corrLength = {corr}
[embedding]
approximate = true
"""


@pytest.fixture(scope="module")
def slot_exe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("slot") / "slot_main"
    inc = os.path.join(ROOT, "parafields-core_b200", "include")
    lib = os.path.join(ROOT, "parafields-core_b200", "lib")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", inc, "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "slot_main.cc"), "-o",
                    str(exe), "-L", lib, "-lpfcuda", "-Wl,-rpath," + lib], check=True)
    return str(exe)


def test_adapter_compiles_in_the_slot(slot_exe):
    assert os.path.exists(slot_exe)


def _ini(tmp_path, **kw):
    p = tmp_path / "f.ini"
    p.write_text(CFG2.format(**kw))
    return str(p)


def _rng_noise(exe, count, seed, out):
    subprocess.run([exe, "noise", str(count), str(seed), str(out)], check=True)
    return np.fromfile(os.path.join(out, "noise.bin"))


def _read(out, name):
    return np.fromfile(os.path.join(out, name))


@pytest.mark.gpu
@pytest.mark.parametrize("cov,aniso,corr,kw", [
    ("exponential", "none", "0.1", dict(corr_length=0.1)),
    ("matern32", "geometric", "0.1 0.02 -0.02 0.06",
     dict(corr_length=(0.1, 0.02, -0.02, 0.06), anisotropy="geometric")),
])
def test_slot_members_against_oracle(slot_exe, oracle, tmp_path, cov, aniso, corr, kw):
    ini = _ini(tmp_path, cov=cov, aniso=aniso, corr=corr)
    r = subprocess.run([slot_exe, "run", ini, "11", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0 and "slot ok" in r.stdout, r.stdout + r.stderr
    d = desc_of(dict(dim=2, cells=(48, 40), covariance=cov, variance=1.3, approximate=True, **kw))
    g = oracle.resolve(d)
    lam, _, _ = oracle.spectrum(d)
    noise = _rng_noise(slot_exe, g.noise, 11, tmp_path)
    field, _ = oracle.generate(d, lam, noise)
    assert rel(_read(tmp_path, "field.bin"), field) < 1e-11
    cx = oracle.matvec(d, lam, pfb200.OP_MUL, field)
    assert rel(_read(tmp_path, "cx.bin"), cx) < 1e-12
    rcx = oracle.matvec(d, lam, pfb200.OP_ROOT, cx)
    assert rel(_read(tmp_path, "rcx.bin"), rcx) < 1e-12
    # multiplyInverse: the reference's innerCG (energy stagnation, cgIterations) through the
    # library, identical to a direct pf_multiply_inverse call on the same right-hand side
    P = pfb200.Plan(d)
    P.spectrum_build()
    x, _ = P.multiply_inverse(_read(tmp_path, "rcx.bin"), mode=pfb200.CG_REFERENCE)
    assert rel(_read(tmp_path, "inv.bin"), x) < 1e-12
    P.close()
    # refineMatrix: the traits double the cells, update() rebuilds the plan at that level
    dr = desc_of(dict(dim=2, cells=(96, 80), covariance=cov, variance=1.3, approximate=True, **kw))
    gr = oracle.resolve(dr)
    lamr, _, _ = oracle.spectrum(dr)
    fr, _ = oracle.generate(dr, lamr, _rng_noise(slot_exe, gr.noise, 11, tmp_path))
    assert rel(_read(tmp_path, "refined_field.bin"), fr) < 1e-11


@pytest.mark.gpu
def test_slot_custom_functor_equals_builtin(slot_exe, oracle, tmp_path):
    """fillMatrix(UserExponential()) on a custom-iso field: the functor is evaluated on the
    host at the matrix cells (ScaledIdentityMatrix geometry), the transform and eigenvalue
    check run on the GPU (pf_spectrum_build_values); the realization equals the built-in
    exponential's on the same noise."""
    ini = _ini(tmp_path, cov="custom-iso", aniso="none", corr="0.1")
    r = subprocess.run([slot_exe, "custom", ini, "5", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    d = desc_of(dict(dim=2, cells=(48, 40), covariance="exponential", variance=1.3, approximate=True,
                     corr_length=0.1))
    g = oracle.resolve(d)
    lam, _, _ = oracle.spectrum(d)
    field, _ = oracle.generate(d, lam, _rng_noise(slot_exe, g.noise, 5, tmp_path))
    assert rel(_read(tmp_path, "field.bin"), field) < 1e-11


@pytest.mark.gpu
def test_slot_custom_without_fillmatrix_throws(slot_exe, tmp_path):
    ini = _ini(tmp_path, cov="custom-iso", aniso="none", corr="0.1")
    r = subprocess.run([slot_exe, "run", ini, "5", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 4
    assert "you need to call fillMatrix with your covariance class as parameter" in r.stdout
