"""C++ facade (parafields-core_b200/include/parafields_b200/randomfield.hh): the
reference's configuration keys and RandomField methods on top of the C ABI.
CPU: key -> descriptor mapping and error messages.  GPU: generate(seed) with the
reference's CppRNGBackend stream, timesMatrix, timesInverseMatrix against the oracle
fed the same noise."""
import os
import subprocess

import numpy as np
import pytest

import pfb200
from helpers import desc_of, rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def facade_exe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("facade") / "facade_main"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "parafields-core_b200", "include"),
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "facade_main.cc"),
                    "-o", str(exe), "-L", os.path.join(ROOT, "parafields-core_b200", "lib"), "-lpfcuda",
                    "-Wl,-rpath," + os.path.join(ROOT, "parafields-core_b200", "lib")], check=True)
    return str(exe)


def write_ini(tmp_path, text):
    p = tmp_path / "field.ini"
    p.write_text(text)
    return str(p)


def test_config_keys(facade_exe, tmp_path):
    ini = write_ini(tmp_path, """
[grid]
cells = 64 32
extensions = 2 1
[stochastic]
variance = 1.5
covariance = gammaExponential
expGamma = 1.2
anisotropy = geometric
corrLength = 0.1 0.02 0.03 0.05
[embedding]
factor = 3
approximate = true
threshold = 1e-12
[randomField]
cgIterations = 50
transform = boxCox
[transform]
boxCoxLambda = 0.25
""")
    out = subprocess.run([facade_exe, "config", ini], capture_output=True, text=True).stdout
    assert "dim=2 cells=64,32,1 ext=2,1,1 factor=3 periodic=0 cov=8 var=1.5 aniso=2 corr=0.1,0.02,0.03,0.05" in out
    assert "approx=1 thr=1e-12 transposed=-1 prec=0 eig=0 cg=50 transform=4 boxcox=0.25 gamma=1.2" in out


@pytest.mark.parametrize("per,extra,want", [
    ("merge", "sigmoid = smooth\nsigmoidStart = 0.5\nmergeRecursions = 3\n[stochastic]\nsigmoidCombine = tensor\n",
     "per=1 sig=1 comb=2 mrec=3 sstart=0.5 send=2"),
    ("fold", "foldMaxFactor = 2\nfoldRecursions = 4\n", "per=2 sig=0 comb=0 mrec=99 sstart=1 send=2 fmf=2 frec=4"),
    ("cofold", "cofoldMaxFactor = 3\ncofoldRecursions = 2\n", "per=3 sig=0 comb=0 mrec=99 sstart=1 send=2 fmf=1 "
     "frec=99 cmf=3 crec=2"),
])
def test_periodization_keys(facade_exe, tmp_path, per, extra, want):
    """embedding.periodization and its sigmoid / merge / fold / cofold keys (matrix.hh:515-579,
    652-1013) reach the descriptor."""
    ini = write_ini(tmp_path, "[grid]\ncells = 16 16\nextensions = 1 1\n[stochastic]\nvariance = 1\ncovariance = exponential\n"
                    "corrLength = 0.1\n[embedding]\nfactor = 3\nperiodization = " + per + "\n" + extra)
    out = subprocess.run([facade_exe, "config", ini], capture_output=True, text=True).stdout
    assert want in out, out


@pytest.mark.parametrize("text,msg", [
    ("grid.cells = 8 8\ngrid.extensions = 1 1\nstochastic.variance = 1\nstochastic.covariance = foo\n"
     "stochastic.corrLength = 0.1\n", "covariance structure foo not known"),
    ("grid.cells = 8 8\ngrid.extensions = 1 1\nstochastic.variance = 1\nstochastic.covariance = exponential\n"
     "stochastic.corrLength = 0.1\nstochastic.anisotropy = weird\n", "stochastic.anisotropy must be"),
    ("grid.cells = 8 8\ngrid.extensions = 1 1\nstochastic.variance = 1\nstochastic.covariance = exponential\n"
     "stochastic.corrLength = 0.1\nrandomField.transform = cube\n", "transform type not known"),
    ("grid.cells = 8 8\ngrid.extensions = 1 1\nstochastic.variance = 1\nstochastic.covariance = exponential\n"
     "stochastic.corrLength = 0.1\nembedding.periodization = twist\n", "stochastic.periodization must be"),
    ("grid.cells = 8 8\ngrid.extensions = 1 1\nstochastic.variance = 1\nstochastic.covariance = exponential\n"
     "stochastic.corrLength = 0.1\nembedding.periodization = cofold\nembedding.sigmoid = step\n",
     "embedding.sigmoid must be"),
])
def test_config_errors(facade_exe, tmp_path, text, msg):
    out = subprocess.run([facade_exe, "config", write_ini(tmp_path, text)], capture_output=True, text=True).stdout
    assert msg in out


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_facade_generate_and_products(facade_exe, tmp_path, oracle, dim):
    if dim == 2:
        keys = "grid.cells = 48 40\ngrid.extensions = 1 1\nstochastic.corrLength = 0.1\n"
        cfg = dict(dim=2, cells=(48, 40), covariance="exponential", corr_length=0.1)
    else:
        keys = "grid.cells = 16 12 10\ngrid.extensions = 1 1 1\nstochastic.anisotropy = axiparallel\n" \
               "stochastic.corrLength = 0.1 0.08 0.05\n"
        cfg = dict(dim=3, cells=(16, 12, 10), covariance="exponential", corr_length=(0.1, 0.08, 0.05))
    ini = write_ini(tmp_path, keys + "stochastic.variance = 1\nstochastic.covariance = exponential\n"
                    "randomField.transform = logNormal\nrandomField.cgIterations = 60\n")
    r = subprocess.run([facade_exe, "run", ini, "17", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    ld = lambda n: np.fromfile(str(tmp_path / n), dtype=np.float64)
    d = desc_of(cfg)
    lam, _, _ = oracle.spectrum(d)
    noise = ld("noise.bin")
    field, _ = oracle.generate(d, lam, noise)
    assert rel(ld("field.bin"), field) < 1e-11
    assert rel(ld("bulk.bin"), np.exp(field)) < 1e-11
    cx = oracle.matvec(d, lam, pfb200.OP_MUL, field)
    assert rel(ld("cx.bin"), cx) < 1e-12
    assert rel(ld("cinvcx.bin"), field) < 1e-6  # C^-1 (C x) = x up to the CG stopping rule
    w = ld("white.bin")
    assert abs(w.mean()) < 0.2 and abs(w.std() - 1) < 0.2


@pytest.mark.gpu
def test_facade_refine_coarsen(facade_exe, tmp_path, oracle):
    """refineMatrix + refine copies every value to its 2^d children; coarsenMatrix + coarsen
    averages them back; with randomField.cacheInvMatvec the refined C x is recomputed as
    2^d C_fine refine(x) from the cached x (randomfield.hh:880-945)."""
    ini = write_ini(tmp_path, "grid.cells = 24 20\ngrid.extensions = 1 1\nstochastic.corrLength = 0.1\n"
                    "stochastic.variance = 1\nstochastic.covariance = exponential\n")
    r = subprocess.run([facade_exe, "refine", ini, "5", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    ld = lambda n: np.fromfile(str(tmp_path / n), dtype=np.float64)
    x = ld("field.bin").reshape(20, 24)
    fine = np.repeat(np.repeat(x, 2, axis=0), 2, axis=1)
    assert np.array_equal(ld("refined.bin").reshape(40, 48), fine)
    assert np.allclose(ld("back.bin").reshape(20, 24), x, rtol=0, atol=1e-15)
    d_fine = desc_of(dict(dim=2, cells=(48, 40), covariance="exponential", corr_length=0.1))
    lam, _, _ = oracle.spectrum(d_fine)
    ref = 4.0 * oracle.matvec(d_fine, lam, pfb200.OP_MUL, fine.ravel())
    assert rel(ld("cached_refined.bin"), ref) < 1e-12


@pytest.mark.gpu
def test_facade_write_and_read_field_files(facade_exe, tmp_path):
    """writeToFile (randomfield.hh:706-713) writes <name>.stoch.h5, <name>.xdmf and <name>.field;
    RandomField(fileName) and RandomField(config, fileName) read the same field back."""
    ini = write_ini(tmp_path, "grid.cells = 24 20 12\ngrid.extensions = 1 1 0.5\nstochastic.variance = 1\n"
                    "stochastic.covariance = exponential\nstochastic.corrLength = 0.1\n")
    r = subprocess.run([facade_exe, "io", ini, "9", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0 and "io ok" in r.stdout, r.stdout + r.stderr
    for ext in (".stoch.h5", ".xdmf", ".field"):
        assert (tmp_path / ("saved" + ext)).exists()
    assert '[ grid ]\ncells = "24 20 12"' in (tmp_path / "saved.field").read_text()
    a = np.fromfile(str(tmp_path / "a.bin"), dtype=np.float64)
    b = np.fromfile(str(tmp_path / "b.bin"), dtype=np.float64)
    assert np.array_equal(a, b)
    field = pfb200.read_field(tmp_path / "saved", (24, 20, 12))
    assert field.size == 24 * 20 * 12 and np.isfinite(field).all()


@pytest.mark.gpu
def test_facade_fftw_measure_and_wisdom(facade_exe, tmp_path, oracle):
    """fftw.measure plans the realization passes by measurement once the matrix exists;
    fftw.useWisdom writes the planning choices to wisdom-R2CField-b200.txt in the working
    directory when the matrix goes away and reads them back for the next one
    (r2cfieldbackend.hh:75-96, 212-216).  The field is the oracle's either way."""
    keys = ("grid.cells = 48 40\ngrid.extensions = 1 1\nstochastic.corrLength = 0.1\nstochastic.variance = 1\n"
            "stochastic.covariance = exponential\nrandomField.cgIterations = 60\n"
            "fftw.measure = true\nfftw.useWisdom = true\n")
    ini = write_ini(tmp_path, keys)
    d = desc_of(dict(dim=2, cells=(48, 40), covariance="exponential", corr_length=0.1))
    lam, _, _ = oracle.spectrum(d)
    for attempt in range(2):  # second run: the wisdom file exists and is read
        r = subprocess.run([facade_exe, "run", ini, "17", str(tmp_path)], capture_output=True, text=True,
                           cwd=str(tmp_path))
        assert r.returncode == 0, r.stdout + r.stderr
        wis = (tmp_path / "wisdom-R2CField-b200.txt").read_text().split("\n")
        assert any(line.startswith("0 ") for line in wis) and any(line.startswith("2 ") for line in wis)
        noise = np.fromfile(str(tmp_path / "noise.bin"), dtype=np.float64)
        field, _ = oracle.generate(d, lam, noise)
        assert rel(np.fromfile(str(tmp_path / "field.bin"), dtype=np.float64), field) < 1e-11
