"""OVF 2.0 files: save_ovf, read_ovf and mag2ovf of src/ovf2.jl, on the
library's native reader and writer (mm_ovf_* in include/mmcuda.h)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_TYPES = {"Float64": _lib.MM_OVF_BINARY8, "Float32": _lib.MM_OVF_BINARY4, "String": _lib.MM_OVF_TEXT,
          np.float64: _lib.MM_OVF_BINARY8, np.float32: _lib.MM_OVF_BINARY4, float: _lib.MM_OVF_BINARY8,
          str: _lib.MM_OVF_TEXT}
_NAMES = {_lib.MM_OVF_BINARY8: "Float64", _lib.MM_OVF_BINARY4: "Float32", _lib.MM_OVF_TEXT: "String"}


def _type_code(t) -> int:
    try:
        return _TYPES[t]
    except (KeyError, TypeError):
        raise ValueError("OVF type must be Float64, Float32 or String") from None


class OVF2:
    """OVF2{T} of src/ovf2.jl:1-13: mesh nodes and steps, data type, title and
    the 3N values (AoS, x fastest)."""

    def __init__(self, xnodes=0, ynodes=0, znodes=0, xstepsize=0.0, ystepsize=0.0, zstepsize=0.0,
                 type="Float64", name="", data=None):
        self.xnodes, self.ynodes, self.znodes = int(xnodes), int(ynodes), int(znodes)
        self.xstepsize, self.ystepsize, self.zstepsize = float(xstepsize), float(ystepsize), float(zstepsize)
        self.type = type
        self.name = name
        n3 = 3 * self.xnodes * self.ynodes * self.znodes
        self.data = np.zeros(n3) if data is None else np.asarray(data, dtype=np.float64).reshape(-1)

    def _desc(self):
        return _lib.MeshDesc(self.xnodes, self.ynodes, self.znodes, self.xstepsize, self.ystepsize,
                             self.zstepsize, 0)


def save_ovf(obj, fname: str, type=None):
    """save_ovf(sim, fname; type=Float64)  src/ovf2.jl:44-62, or
    save_ovf(ovf::OVF2, fname; type=ovf.type)  :70-78."""
    L = _lib.load()
    if isinstance(obj, OVF2):
        code = _type_code(obj.type if type is None else type)
        data = np.ascontiguousarray(obj.data, dtype=np.float64)
        if data.size != 3 * obj.xnodes * obj.ynodes * obj.znodes:
            raise ValueError("OVF2 data does not match xnodes*ynodes*znodes")
        d = obj._desc()
        _lib.check(L.mm_ovf_write(fname.encode(), ctypes.byref(d), _lib.dptr(data), code, obj.name.encode()))
        return
    code = _type_code("Float64" if type is None else type)
    _lib.check(L.mm_save_ovf(obj._h.h, fname.encode(), code, str(obj.name).encode()))


def read_ovf(arg, fname: str | None = None):
    """read_ovf(fname) -> OVF2  src/ovf2.jl:246-291, or read_ovf(sim, fname)
    :197-208, which sets the Sim's m from the file."""
    L = _lib.load()
    if fname is not None:
        _lib.check(L.mm_load_ovf(arg._h.h, fname.encode()))
        return None
    d = _lib.MeshDesc()
    code = ctypes.c_int()
    title = ctypes.create_string_buffer(4096)
    _lib.check(L.mm_ovf_read_header(arg.encode(), ctypes.byref(d), ctypes.byref(code), title, 4096))
    n = d.nx * d.ny * d.nz
    data = np.empty(3 * n)
    _lib.check(L.mm_ovf_read(arg.encode(), _lib.dptr(data), n))
    return OVF2(d.nx, d.ny, d.nz, d.dx, d.dy, d.dz, _NAMES[code.value], title.value.decode(errors="replace"),
                data)


def mag2ovf(m, nx: int, ny: int, nz: int, dx=1e-9, dy=1e-9, dz=1e-9, fname="mag", type="Float64"):
    """mag2ovf(m, nx, ny, nz; dx, dy, dz, fname, type)  src/ovf2.jl:293-343."""
    save_ovf(OVF2(nx, ny, nz, dx, dy, dz, type, fname, m), fname)
