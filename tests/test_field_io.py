"""Field files (randomfield.hh:706-713, stochastic.hh:80-110 / 273-294, io.hh:170-349): the
field as dataset /stochastic of <name>.stoch.h5, <name>.xdmf, the configuration as
<name>.field.  The HDF5 file is written without libhdf5; besides the library's own reader,
these tests parse it with an independent reader of the HDF5 structures (superblock v0,
symbol-table root group, version 1 object headers, contiguous layout)."""
import os
import struct
import subprocess

import numpy as np
import pytest

import pfb200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def h5_exe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("h5") / "h5_main"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "parafields-core_b200", "include"),
                    os.path.join(ROOT, "tests", "cpp", "h5_main.cc"), "-o", str(exe)], check=True)
    return str(exe)


def parse_h5(path, name="stochastic"):
    """Independent reader: superblock v0 -> root object header -> symbol table message ->
    B-tree (group node, level 0) -> symbol table node -> dataset object header ->
    dataspace / datatype / layout -> data."""
    b = open(path, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    assert b[8] == 0 and b[13] == 8 and b[14] == 8
    leaf_k, internal_k = struct.unpack_from("<HH", b, 16)
    base, free, eof, drv = struct.unpack_from("<QQQQ", b, 24)
    assert base == 0 and free == 2 ** 64 - 1 and drv == 2 ** 64 - 1 and eof == len(b)
    _, root_oh, cache = struct.unpack_from("<QQI", b, 56)
    assert cache == 1

    def messages(addr):
        ver, n, refc, size = struct.unpack_from("<BxHII", b, addr)
        assert ver == 1 and refc == 1 and size % 8 == 0
        out, p = [], addr + 16
        for _ in range(n):
            t, s, _flags = struct.unpack_from("<HHB", b, p)
            assert s % 8 == 0
            out.append((t, b[p + 8:p + 8 + s]))
            p += 8 + s
        assert p == addr + 16 + size
        return out

    st = [m for t, m in messages(root_oh) if t == 0x11]
    assert len(st) == 1
    btree, heap = struct.unpack_from("<QQ", st[0], 0)
    assert struct.unpack_from("<QQ", b, 80) == (btree, heap)
    assert b[heap:heap + 4] == b"HEAP"
    hsize, hfree, hdata = struct.unpack_from("<QQQ", b, heap + 8)
    assert hfree == 1 and b[hdata] == 0
    assert b[btree:btree + 4] == b"TREE" and b[btree + 4] == 0 and b[btree + 5] == 0
    used = struct.unpack_from("<H", b, btree + 6)[0]
    assert used == 1
    k0, snod, k1 = struct.unpack_from("<QQQ", b, btree + 24)
    assert btree + 24 + 2 * internal_k * 8 + (2 * internal_k + 1) * 8 <= len(b)
    assert b[snod:snod + 4] == b"SNOD" and b[snod + 4] == 1
    nsym = struct.unpack_from("<H", b, snod + 6)[0]
    assert nsym == 1 and snod + 8 + 2 * leaf_k * 40 <= len(b)
    name_off, dset_oh = struct.unpack_from("<QQ", b, snod + 8)
    got = b[hdata + name_off:b.index(b"\0", hdata + name_off)].decode()
    assert got == name and name_off == k1 and k0 == 0
    dims = fmt = addr = size = None
    for t, m in messages(dset_oh):
        if t == 1:
            assert m[0] == 1 and m[2] == 0
            dims = list(struct.unpack_from("<%dQ" % m[1], m, 8))
        elif t == 3:
            assert m[0] == 0x11 and m[1] == 0x20
            esz = struct.unpack_from("<I", m, 4)[0]
            off, prec, eloc, esize, mloc, msize, bias = struct.unpack_from("<HHBBBBI", m, 8)
            assert (esz, m[2], prec, eloc, esize, mloc, msize, bias) in (
                (8, 63, 64, 52, 11, 0, 52, 1023), (4, 31, 32, 23, 8, 0, 23, 127))
            fmt = "<d" if esz == 8 else "<f"
        elif t == 8:
            assert m[0] == 3 and m[1] == 1
            addr, size = struct.unpack_from("<QQ", m, 2)
    n = int(np.prod(dims))
    assert size == n * struct.calcsize(fmt) and addr % 8 == 0 and addr + size == len(b)
    return dims, np.frombuffer(b, dtype=fmt, count=n, offset=addr)


@pytest.mark.parametrize("dim,cells,ext,f32", [
    (1, (37,), (2.0,), False), (2, (12, 7), (1.0, 0.5), False), (3, (5, 4, 3), (1.0, 2.0, 3.0), True)])
def test_stoch_h5_roundtrip_and_structure(h5_exe, tmp_path, dim, cells, ext, f32):
    base = str(tmp_path / "field")
    args = [h5_exe, "write", base, str(dim)] + [str(c) for c in cells] + [str(e) for e in ext] + (["f32"] if f32 else [])
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    dims, vals = parse_h5(base + ".stoch.h5")
    assert dims == list(reversed(cells))  # io.hh:203-205
    i = np.arange(int(np.prod(cells)))
    want = np.sin(0.37 * i) * 1.5 + 1e-3 * i
    if f32:
        want = want.astype(np.float32).astype(np.float64)
    assert np.array_equal(vals, want)  # stored as F64LE either way (io.hh:9, 218-224)
    xdmf = open(base + ".xdmf").read()
    rev = " ".join(str(c) for c in reversed(cells)) + " "
    assert f'NumberOfElements="{rev}"' in xdmf and f'<DataItem Dimensions="{rev}" Format="HDF">' in xdmf
    assert base + ".stoch.h5:/stochastic" in xdmf and xdmf.startswith('<?xml version="1.0" ?>')


def test_stoch_h5_reader_errors(h5_exe, tmp_path):
    base = str(tmp_path / "f")
    r = subprocess.run([h5_exe, "read", base, "2", "4", "4"], capture_output=True, text=True)
    assert r.returncode == 1 and "File is missing: " + base + ".stoch.h5" in r.stdout
    subprocess.run([h5_exe, "write", base, "2", "4", "3", "1", "1"], check=True, capture_output=True)
    r = subprocess.run([h5_exe, "read", base, "2", "3", "4"], capture_output=True, text=True)
    assert r.returncode == 1 and "does not hold the configured cells" in r.stdout
    r = subprocess.run([h5_exe, "read", base, "2", "4", "3"], capture_output=True, text=True)
    assert r.returncode == 0 and len(r.stdout.split()) == 12


def test_field_config_report_roundtrip(h5_exe, tmp_path):
    ini = tmp_path / "c.ini"
    ini.write_text("[grid]\ncells = 16 8\nextensions = 1 0.5\n[stochastic]\ncovariance = exponential\n"
                   "corrLength = 0.1\nvariance = 1\n[embedding]\nperiodization = fold\n[randomField]\n"
                   "transform = logNormal\n")
    r = subprocess.run([h5_exe, "report", str(ini)], capture_output=True, text=True)
    assert r.returncode == 0
    assert '[ grid ]\ncells = "16 8"\nextensions = "1 0.5"\n' in r.stdout
    assert '[ stochastic ]\ncorrLength = "0.1"\ncovariance = "exponential"\nvariance = "1"\n' in r.stdout


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_c_abi_field_files_host(tmp_path, dtype):
    cells = (6, 5, 4)
    x = (np.random.default_rng(1).standard_normal(int(np.prod(cells)))).astype(dtype)
    base = tmp_path / "g"
    pfb200.write_field(base, x, cells, (1.0, 1.0, 2.0))
    dims, vals = parse_h5(str(base) + ".stoch.h5")
    assert dims == [4, 5, 6] and np.array_equal(vals, x.astype(np.float64))
    y = pfb200.read_field(base, cells, precision=pfb200.PREC_F64 if dtype == np.float64 else pfb200.PREC_F32)
    assert y.dtype == dtype and np.array_equal(y, x)
    with pytest.raises(pfb200.PfError) as e:
        pfb200.read_field(tmp_path / "nothing", cells)
    assert e.value.status == pfb200.PF_ERR_IO and "File is missing" in str(e.value)
    with pytest.raises(pfb200.PfError) as e:
        pfb200.read_field(base, (5, 6, 4))
    assert e.value.status == pfb200.PF_ERR_IO


@pytest.mark.gpu
def test_c_abi_field_files_device(tmp_path):
    import torch
    cells = (32, 24, 16)
    x = torch.randn(int(np.prod(cells)), dtype=torch.float32, device="cuda")
    base = tmp_path / "d"
    pfb200.write_field(base, x, cells, (1.0, 1.0, 1.0))
    y = torch.empty_like(x)
    pfb200.read_field(base, cells, out=y)
    assert torch.equal(x, y)
    _, vals = parse_h5(str(base) + ".stoch.h5")
    assert np.array_equal(vals, x.cpu().numpy().astype(np.float64))
