"""OVF 2.0 reader / writer of the library (host-only, no GPU): the cases of
test/test_ovf.jl plus a byte-level check of the binary layout against an
independent numpy parser."""
import os

import numpy as np
import pytest

from mmcuda import _lib
from mmcuda.ovf import OVF2, mag2ovf, read_ovf, save_ovf

M = np.array([0.6, 0.8, 0, 0.6, 0.8, 0])


@pytest.mark.parametrize("fname,type", [("Float64", "Float64"), ("Float32", "Float32"), ("String", "String")])
def test_ovf(tmp_path, fname, type):
    """test_ovf  test/test_ovf.jl:8-65 at file level (the Sim-level calls run
    in test_gpu_api.py)."""
    path = str(tmp_path / fname)
    save_ovf(OVF2(2, 1, 1, 1e-9, 1e-9, 1e-9, type, "saving", M), path)
    ovf = read_ovf(path)  # test_reading
    assert len(ovf.data) == 6
    assert np.max(np.abs(ovf.data - M)) < 1e-6
    assert ovf.type == type and (ovf.xnodes, ovf.ynodes, ovf.znodes) == (2, 1, 1)
    assert ovf.name == "saving" and ovf.xstepsize == 1e-9
    save_ovf(ovf, path + "_copy_float64")  # test_copying
    ovf2 = read_ovf(path + "_copy_float64")
    assert len(ovf2.data) == 6 and np.max(np.abs(ovf2.data - M)) < 1e-6
    save_ovf(read_ovf(path), path + "_copy_string", type="String")
    ovf3 = read_ovf(path + "_copy_string")
    assert ovf3.type == "String" and np.max(np.abs(ovf3.data - M)) < 1e-6


def test_mag2ovf(tmp_path):
    """test_mag2ovf  test/test_ovf.jl:46-55."""
    f = str(tmp_path / "test")
    mag2ovf(M, 2, 1, 1, fname=f)
    ovf = read_ovf(f)
    assert np.allclose(ovf.data, M, atol=1e-6)
    assert (ovf.xnodes, ovf.ynodes, ovf.znodes) == (2, 1, 1)
    assert os.path.exists(f + ".ovf")


def test_text_round_trip_is_exact(tmp_path):
    """Text values are written as shortest round-trip decimals."""
    rng = np.random.default_rng(11)
    m = rng.normal(size=3 * 24)
    f = str(tmp_path / "t")
    save_ovf(OVF2(4, 3, 2, 2e-9, 2e-9, 1e-9, "String", "t", m), f)
    np.testing.assert_array_equal(read_ovf(f).data, m)


def _parse_binary(path):
    """Independent reader: header lines up to the data marker, then the raw block."""
    raw = open(path, "rb").read()
    hdr, pos = {}, 0
    while True:
        end = raw.index(b"\n", pos)
        line = raw[pos:end].decode()
        pos = end + 1
        if line.startswith("# ") and ":" in line:
            k, v = line[2:].split(":", 1)
            hdr[k.strip()] = v.strip()
            if k.strip() == "Begin" and v.strip().startswith("Data"):
                return hdr, raw, pos


@pytest.mark.parametrize("kind,dt,chk", [("Float64", "<f8", 123456789012345.0), ("Float32", "<f4", 1234567.0)])
def test_binary_layout(tmp_path, kind, dt, chk):
    nx, ny, nz = 5, 3, 2
    rng = np.random.default_rng(7)
    m = rng.normal(size=(nz, ny, nx, 3))
    m /= np.linalg.norm(m, axis=-1, keepdims=True)
    f = str(tmp_path / "lay.ovf")
    save_ovf(OVF2(nx, ny, nz, 2e-9, 2.5e-9, 3e-9, kind, "lay", m.reshape(-1)), f)
    hdr, raw, pos = _parse_binary(f)
    assert hdr["Title"] == "lay" and hdr["meshunit"] == "m" and hdr["valuelabels"] == "m_x m_y m_z"
    assert hdr["xnodes"] == "5" and hdr["ynodes"] == "3" and hdr["znodes"] == "2"
    assert float(hdr["xstepsize"]) == 2e-9 and float(hdr["zstepsize"]) == 3e-9
    assert float(hdr["xmax"]) == 5 * 2e-9 and float(hdr["xbase"]) == 1e-9
    w = np.dtype(dt).itemsize
    assert hdr["valuedim"] == "3" and hdr["Begin"] == "Data Binary %d" % w
    block = np.frombuffer(raw, dtype=dt, count=1 + 3 * nx * ny * nz, offset=pos)
    assert block[0] == chk
    np.testing.assert_array_equal(block[1:], m.reshape(-1).astype(dt))  # x fastest, components together
    tail = raw[pos + w * (1 + 3 * nx * ny * nz):].decode()
    assert tail == "\n# End: Data Binary %d\n# End: Segment\n" % w


def test_errors(tmp_path):
    L = _lib.load()
    f = tmp_path / "bad.ovf"
    f.write_text("# OOMMF OVF 1.0\n")
    d = _lib.MeshDesc()
    assert L.mm_ovf_read_header(str(f).encode(), d, None, None, 0) == _lib.MM_ERR_ARG
    assert "not a OVF2" in _lib.last_error()
    save_ovf(OVF2(2, 1, 1, 1e-9, 1e-9, 1e-9, "Float64", "x", M), str(tmp_path / "ok"))
    out = np.empty(9)
    assert L.mm_ovf_read(str(tmp_path / "ok").encode(), _lib.dptr(out), 3) == _lib.MM_ERR_ARG
    assert "does not match" in _lib.last_error()
    trunc = tmp_path / "short.ovf"
    trunc.write_bytes(open(str(tmp_path / "ok.ovf"), "rb").read()[:-60])
    assert L.mm_ovf_read(str(trunc).encode(), _lib.dptr(out), 2) == _lib.MM_ERR_ARG
    with pytest.raises(ValueError):
        save_ovf(OVF2(2, 1, 1, 1e-9, 1e-9, 1e-9, "Float16", "x", M), str(tmp_path / "t"))


def test_oversized_header_refused(tmp_path):
    """Node counts whose product (times 3 values a cell) overflows int64 are
    refused while parsing the header, before any product is formed."""
    L = _lib.load()
    ok = str(tmp_path / "ok")
    save_ovf(OVF2(2, 1, 1, 1e-9, 1e-9, 1e-9, "String", "x", M), ok)
    text = open(ok + ".ovf").read()
    for nodes in (("2000000000", "2000000000", "2000000000"), ("2147483647", "2147483647", "2")):
        bad = text.replace("# xnodes: 2\n", "# xnodes: %s\n" % nodes[0])
        bad = bad.replace("# ynodes: 1\n", "# ynodes: %s\n" % nodes[1]).replace("# znodes: 1\n", "# znodes: %s\n" % nodes[2])
        assert bad != text
        f = tmp_path / "huge.ovf"
        f.write_text(bad)
        d = _lib.MeshDesc()
        assert L.mm_ovf_read_header(str(f).encode(), d, None, None, 0) == _lib.MM_ERR_ARG
        assert "too large" in _lib.last_error()
        out = np.empty(6)
        assert L.mm_ovf_read(str(f).encode(), _lib.dptr(out), 2) == _lib.MM_ERR_ARG
