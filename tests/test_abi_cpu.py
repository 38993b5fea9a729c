"""CPU-side checks of the product: the C-ABI library builds for sm_100a, loads,
exports every symbol that include/mmcuda.h declares, and the host-side
mirror of the reference API behaves like the reference without a GPU."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mmcuda.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^int\s+(mm_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_header_symbol():
    from mmcuda import _lib

    L = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == syms
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT\s+(mm_\w+)", out))
    assert set(syms) <= exported


def test_library_is_sm100a():
    from mmcuda import _lib

    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    assert "sm_100a" in out


def test_abi_version_and_error_path():
    from mmcuda import _lib

    L = _lib.load()
    assert L.mm_abi_version() == 1
    # a null handle is rejected with MM_ERR_ARG and a message, no GPU needed
    rc = L.mm_synchronize(None)
    assert rc == -1
    assert "null handle" in _lib.last_error()
    rc = L.mm_create(None, 0, 0, None)
    assert rc == -1


def test_padded_lengths_match_convolution_rule():
    """Any padded length P >= 2n-1 gives the reference's linear convolution;
    the library picks the smallest 7-smooth one (even along x)."""

    def smooth(p):
        for f in (2, 3, 5, 7):
            while p % f == 0:
                p //= f
        return p == 1

    def padded(n, even):
        if n <= 1:
            return 1
        p = 2 * n - 1
        while not smooth(p) or (even and p % 2):
            p += 1
        return p

    assert padded(1, True) == 1
    assert padded(2, True) == 4 and padded(2, False) == 3
    assert padded(256, True) == 512 and padded(64, False) == 128 and padded(1024, True) == 2048
    assert padded(200, True) == 400 and padded(50, False) == 100
    assert padded(251, True) == 504
    for n in range(1, 300):
        assert padded(n, False) >= 2 * n - 1


def test_host_field_initialisers_follow_reference():
    from mmcuda.sim import FDMesh, _normalise, _scalar_field, _vector_field

    mesh = FDMesh(nx=3, ny=2, nz=2, dx=2e-9)
    # f(i,j,k,dx,dy,dz) with 1-based indices, x fastest (src/helper.jl:14-22)
    a = _scalar_field(mesh, lambda i, j, k, dx, dy, dz: 100 * k + 10 * j + i)
    assert a[0] == 111 and a[1] == 112 and a[3] == 121 and a[6] == 211
    v = _vector_field(mesh, (1, 2, 2))
    _normalise(v)
    assert np.allclose(v.reshape(-1, 3), [1 / 3, 2 / 3, 2 / 3])
    z = np.zeros(3 * mesh.n_total)
    _normalise(z)  # |m|^2 == 0 stays 0 (src/helper.jl:262)
    assert not np.isnan(z).any()
