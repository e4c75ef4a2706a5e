"""The profiling driver's wisdom text (parafields-core_b200/pass_profile.py): one entry per
realization pass with the keys the library's measured planning uses, and the pseudo-pass 3
entry with the plane groups; accepted by pf_wisdom_import (host only, no GPU)."""
import os
import sys
from types import SimpleNamespace

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "parafields-core_b200"))
import pass_profile  # noqa: E402


def info(dim, cells, torus, prec=1):
    return SimpleNamespace(dim=dim, cells=list(cells) + [1] * (3 - dim), ext_cells=list(torus) + [1] * (3 - dim),
                           precision=prec)


def test_wisdom_lines_3d():
    text = pass_profile.wisdom_lines(info(3, (256, 256, 256), (512, 512, 512)), {1: (2, 0), 2: (0, 3)}, 4)
    assert text.splitlines() == ["0 512 257 512 1 0 0", "1 512 257 256 1 2 0", "2 512 65536 1 1 0 3",
                                 "3 512 257 512 1 0 4"]


def test_wisdom_lines_2d():
    text = pass_profile.wisdom_lines(info(2, (512, 384), (1024, 768), prec=0), {}, 1)
    assert text.splitlines() == ["0 768 513 1 0 0 0", "2 1024 384 1 0 0 0", "3 768 513 1 0 0 1"]


def test_parse_run():
    assert pass_profile.parse_run("2=2,1=0:3,G=8") == ({2: (2, 0), 1: (0, 3)}, 8)


def test_wisdom_text_is_accepted():
    pfb200 = pytest.importorskip("pfb200")
    try:
        pfb200.lib()
    except (RuntimeError, OSError) as e:
        pytest.skip(str(e))
    text = pass_profile.wisdom_lines(info(3, (16, 8, 12), (32, 16, 24)), {0: (1, 2)}, 3)
    pfb200.wisdom_forget()
    pfb200.wisdom_import(text)
    assert sorted(pfb200.wisdom_export().strip().splitlines()) == sorted(text.strip().splitlines())
    pfb200.wisdom_forget()
