"""CPU-side checks of the C ABI: the library loads, exports every function declared
in include/parafields_b200.h, the ctypes mirrors have the C layout, and the
descriptor defaults are the reference's."""
import ctypes as C
import os
import re
import subprocess

import pytest

import pfb200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "parafields_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    if not os.path.exists(pfb200.LIB_PATH):
        pytest.fail("libpfcuda.so not built")
    L = C.CDLL(pfb200.LIB_PATH)
    missing = [f for f in declared_functions() if not hasattr(L, f)]
    assert not missing, missing
    assert len(declared_functions()) >= 15


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "parafields_b200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(pf_field_desc), '
                   'sizeof(pf_eig_stats), sizeof(pf_plan_info), sizeof(pf_cg_opts), sizeof(pf_cg_report), '
                   'sizeof(pf_kernel_time), offsetof(pf_field_desc, boxcox_lambda), '
                   'offsetof(pf_field_desc, cofold_max_factor), sizeof(pf_peaks));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    exp = [C.sizeof(pfb200.FieldDesc), C.sizeof(pfb200.EigStats), C.sizeof(pfb200.PlanInfo),
           C.sizeof(pfb200.CgOpts), C.sizeof(pfb200.CgReport), C.sizeof(pfb200.KernelTime),
           pfb200.FieldDesc.boxcox_lambda.offset, pfb200.FieldDesc.cofold_max_factor.offset,
           C.sizeof(pfb200.Peaks)]
    assert got == exp


def test_descriptor_defaults():
    L = pfb200.lib()
    d = pfb200.FieldDesc()
    L.pf_field_desc_init(C.byref(d))
    assert d.embedding_factor == 2 and d.threshold == 1e-14 and d.cg_iterations == 100
    assert d.transposed == -1 and d.matrix_backend == -1 and d.field_backend == -1
    assert L.pf_version().decode().startswith("parafields-b200")


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(pfb200.PfError) as e:
        pfb200.Plan(pfb200.make_desc(dim=2, cells=(8, 8)))
    assert e.value.status == pfb200.PF_ERR_CUDA
