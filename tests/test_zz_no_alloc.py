"""mm_energy_noalloc: energies without any device allocation by the library.

Some callers cannot call cudaMalloc where they need energies -- a host whose
own pool allocator must own all device memory, a latency-critical loop where
cudaMalloc's implicit device synchronisation is not acceptable, or code that
holds no handle.  This entry point takes device pointers to m, Ms and a
6-double output and keeps its per-block partial sums in a static device array
of the library.  Its result must match the handle-based mm_energy (which
allocates its reduction buffer) on two calls in a row, since the static array
keeps the previous call's contents.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # FP64 on both paths; only the summation order differs


def _setup(nx, ny, nz, pbc, seed):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mmcuda import _lib

    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    Ms = rng.uniform(4e5, 9e5, n)
    Ms[rng.random(n) < 0.1] = 0.0
    m = rng.normal(size=(n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    m[Ms == 0] = 0.0
    A, D, Ku, axis, H = 1.2e-11, 2.5e-3, 3e5, (0.3, -0.2, 0.9), (1.5e4, -2.0e4, 3.0e4)
    bits = (1 if "x" in pbc else 0) | (2 if "y" in pbc else 0) | (4 if "z" in pbc else 0)
    h = _lib.Handle(nx, ny, nz, 2e-9, 2.5e-9, 3e-9, bits, _lib.MM_FP64)
    h.call("mm_set_Ms", _lib.dptr(np.ascontiguousarray(Ms)), 0.0)
    h.set_m(m.reshape(-1))
    h.call("mm_add_exch", None, A, A, A)
    h.call("mm_add_dmi_bulk", D, D, D)
    h.call("mm_add_anis", None, Ku, *axis)
    h.call("mm_add_zeeman", None, *H)
    ref = np.zeros(6)
    tot = ctypes.c_double()
    h.call("mm_energy", _lib.dptr(ref), ctypes.byref(tot))
    dev = torch.device("cuda", 0)
    m_soa = torch.from_numpy(np.ascontiguousarray(m.T)).to(dev)  # [mx..., my..., mz...]
    Ms_d = torch.from_numpy(Ms).to(dev)
    out = torch.zeros(6, dtype=torch.float64, device=dev)
    desc = _lib.MeshDesc(nx, ny, nz, 2e-9, 2.5e-9, 3e-9, bits)
    args = (ctypes.byref(desc), ctypes.c_void_p(m_soa.data_ptr()), ctypes.c_void_p(Ms_d.data_ptr()), A, D, Ku,
            *axis, *H, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    return torch, _lib, h, ref, out, args


@pytest.mark.parametrize("mesh", [(37, 23, 5, ""), (64, 64, 1, "xy"), (16, 8, 12, "xyz")])
def test_energy_noalloc_matches_handle(mesh):
    torch, _lib, h, ref, out, args = _setup(*mesh, seed=mesh[0] * 10000 + mesh[1] * 100 + mesh[2])
    L = _lib.load()
    for call in range(2):  # the static scratch keeps the last call's contents
        out.fill_(float("nan"))
        _lib.check(L.mm_energy_noalloc(*args))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        for t in (0, 1, 2, 4):  # zeeman, exchange, bulk DMI, anisotropy
            assert abs(got[t] - ref[t]) <= REL_TOL * abs(ref[t]), (call, t, got[t], ref[t])
        assert got[3] == 0.0 and got[5] == 0.0
    h.close()


def test_energy_noalloc_rejects_oversized_mesh():
    torch, _lib, h, ref, out, args = _setup(8, 8, 2, "", seed=3)
    big = _lib.MeshDesc(4096, 4096, 2, 2e-9, 2e-9, 2e-9, 0)  # 2^25 cells > 2^24
    rc = _lib.load().mm_energy_noalloc(ctypes.byref(big), *args[1:])
    assert rc == -1 and "static scratch limit" in _lib.last_error()
    h.close()


@pytest.mark.parametrize("mesh", [(37, 23, 5, ""), (16, 8, 12, "xyz")])
def test_energy_noalloc_matches_oracle(mesh):
    """The same energies against the CPU oracle's compute_system_energy
    restatement (src/micro/field.jl:520-536), term by term."""
    from oracle.oracle import OracleSim

    nx, ny, nz, pbc = mesh
    torch, _lib, h, ref, out, args = _setup(*mesh, seed=mesh[0] * 10000 + mesh[1] * 100 + mesh[2])
    rng = np.random.default_rng(mesh[0] * 10000 + mesh[1] * 100 + mesh[2])
    n = nx * ny * nz
    Ms = rng.uniform(4e5, 9e5, n)
    Ms[rng.random(n) < 0.1] = 0.0
    m = rng.normal(size=(n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    m[Ms == 0] = 0.0
    A, D, Ku, axis, H = 1.2e-11, 2.5e-3, 3e5, (0.3, -0.2, 0.9), (1.5e4, -2.0e4, 3.0e4)
    o = OracleSim(nx, ny, nz, 2e-9, 2.5e-9, 3e-9, pbc)
    o.set_Ms(Ms)
    o.set_m(m.reshape(-1))
    o.add_zeeman(np.tile(np.asarray(H), n))
    o.add_exch(Ax=A, Ay=A, Az=A)
    o.add_dmi_bulk(D, D, D)
    o.add_anis(np.full(n, Ku), axis)
    _, per = o.energy(4)  # zeeman, exchange, bulk DMI, anisotropy in the order added
    L = _lib.load()
    _lib.check(L.mm_energy_noalloc(*args))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for t, e in zip((0, 1, 2, 4), per):
        assert abs(got[t] - e) <= REL_TOL * abs(e), (t, got[t], e)
    h.close()


def test_energy_noalloc_allocates_nothing():
    """After the first call (which loads the library's device code and its
    static array), further calls leave the device's free memory unchanged."""
    torch, _lib, h, ref, out, args = _setup(37, 23, 5, "", seed=77)
    L = _lib.load()
    _lib.check(L.mm_energy_noalloc(*args))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        _lib.check(L.mm_energy_noalloc(*args))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    h.close()
