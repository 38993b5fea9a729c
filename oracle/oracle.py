"""ctypes wrapper of the CPU FP64 oracle (``mm_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke()``
and by ``bench.py``'s CPU-baseline leg, as the checker.  The product package
never imports it.

The oracle restates the MicroMagnetic.jl finite-difference path (see the
file:line citations in ``mm_oracle.cpp``).  Arrays are AoS float64
``[mx1, my1, mz1, mx2, ...]`` with x fastest, as in the reference.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libmmoracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP) if needed."""
    src = os.path.join(_HERE, "mm_oracle.cpp")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-s", "libmmoracle.so"], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        vp = ctypes.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [ctypes.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_Ms.argtypes = [vp, _dp]
        L.orc_set_m.argtypes = [vp, _dp]
        L.orc_get_m.argtypes = [vp, _dp]
        L.orc_get_y_current.argtypes = [vp, _dp]
        L.orc_set_pins.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8)]
        L.orc_set_llg.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.orc_add_zeeman.argtypes = [vp, _dp]
        L.orc_add_exch.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_add_dmi_bulk.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_add_dmi_interfacial.argtypes = [vp, _dp]
        L.orc_add_anis.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_add_demag.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_demag_tensor.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [ctypes.c_int] * 4 + [_dp]
        L.orc_set_reference_tensor.argtypes = [ctypes.c_int]
        L.orc_newell_fn.argtypes = [ctypes.c_int] + [ctypes.c_int64] * 3 + [ctypes.c_double] * 3 + [_dp]
        L.orc_term_field.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp]
        L.orc_effective_field.argtypes = [vp, _dp, _dp]
        L.orc_llg_rhs.argtypes = [vp, _dp, _dp]
        L.orc_energy.argtypes = [vp, _dp]
        L.orc_energy.restype = ctypes.c_double
        L.orc_rk4.argtypes = [vp, ctypes.c_double, ctypes.c_int64]
        L.orc_heun.argtypes = [vp, ctypes.c_double, ctypes.c_int64]
        L.orc_set_method.argtypes = [vp, ctypes.c_int]
        L.orc_rk4_time.argtypes = [vp]
        L.orc_rk4_time.restype = ctypes.c_double
        L.orc_dopri_set.argtypes = [vp, ctypes.c_double]
        L.orc_run_until.argtypes = [vp, ctypes.c_double, _dp]
        L.orc_dopri_advance.argtypes = [vp, _dp]
        L.orc_relax.argtypes = [vp, ctypes.c_int, ctypes.c_int64, ctypes.c_double, _dp]
        L.orc_relax.restype = ctypes.c_int64
        d = ctypes.c_double
        L.orc_add_dmi_bulk_spatial.argtypes = [vp, _dp, _dp, _dp]
        L.orc_add_sot.argtypes = [vp, _dp, d, d, d, d]
        L.orc_add_stt_zhang_li.argtypes = [vp, _dp, _dp, d]
        L.orc_add_stt_slonczewski.argtypes = [vp, _dp, d, d, d, d, d, d, d]
        L.orc_add_thermal_noise.argtypes = [vp, _dp, d, d, d, ctypes.c_uint64, d]
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.orc_philox.argtypes = [u32p, u32p, u32p]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def demag_tensor(nx, ny, nz, dx, dy, dz, Nx=0, Ny=0, Nz=0, accurate=True) -> np.ndarray:
    """Real-space Newell tensor, shape (6, N) in order xx yy zz xy xz yz.
    accurate=True: near field in binary128 (correctly rounded entries);
    False: the reference's FP64 arithmetic."""
    n = nx * ny * nz
    out = np.zeros((6, n))
    lib().orc_demag_tensor(nx, ny, nz, dx, dy, dz, Nx, Ny, Nz, 1 if accurate else 0, _ptr(out))
    return out


def reference_tensor_arithmetic(on: bool) -> None:
    """Newell tensor of the following add_demag calls in the reference's FP64
    arithmetic (True) or with the binary128 near field (False, the default)."""
    lib().orc_set_reference_tensor(1 if on else 0)


def newell_fn(c, X, Y, Z, dx, dy, dz):
    """f (c = 0..2) or g (c = 3..5) of tensor component c at the integer
    offset (X, Y, Z) times the normalised cell, in binary128: (hi, lo)."""
    out = np.zeros(2)
    lib().orc_newell_fn(c, X, Y, Z, dx, dy, dz, _ptr(out))
    return out[0], out[1]


class OracleSim:
    """One oracle simulation (mesh + terms + integrator state)."""

    def __init__(self, nx, ny, nz, dx, dy, dz, pbc=""):
        bits = (1 if "x" in pbc else 0) | (2 if "y" in pbc else 0) | (4 if "z" in pbc else 0)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz
        self.h = lib().orc_create(nx, ny, nz, dx, dy, dz, bits)
        if not self.h:
            raise ValueError(lib().orc_last_error().decode())

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.orc_destroy(h)
            self.h = None

    def _vec(self, v, k):
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), (self.n * k,)) if np.ndim(v) == 0 else np.asarray(v, dtype=np.float64).reshape(-1))
        assert a.size == self.n * k
        return a

    def set_Ms(self, Ms):
        a = self._vec(Ms, 1)
        lib().orc_set_Ms(self.h, _ptr(a))

    def set_m(self, m):
        a = np.ascontiguousarray(np.asarray(m, dtype=np.float64).reshape(-1))
        assert a.size == 3 * self.n
        lib().orc_set_m(self.h, _ptr(a))

    def get_m(self):
        out = np.zeros(3 * self.n)
        lib().orc_get_m(self.h, _ptr(out))
        return out

    def set_pins(self, pins):
        a = np.ascontiguousarray(np.asarray(pins, dtype=np.uint8).reshape(-1))
        lib().orc_set_pins(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))

    def set_llg(self, alpha, gamma, precession=True):
        lib().orc_set_llg(self.h, float(alpha), float(gamma), 1 if precession else 0)

    def add_zeeman(self, H):
        H = np.asarray(H, dtype=np.float64)
        if H.size == 3:
            H = np.tile(H, self.n)
        a = np.ascontiguousarray(H.reshape(-1))
        return lib().orc_add_zeeman(self.h, _ptr(a))

    def add_exch(self, A=None, Ax=0.0, Ay=0.0, Az=0.0):
        a = None if A is None else self._vec(A, 1)
        return lib().orc_add_exch(self.h, _ptr(a), Ax, Ay, Az)

    def add_dmi_bulk(self, Dx, Dy, Dz):
        return lib().orc_add_dmi_bulk(self.h, Dx, Dy, Dz)

    def add_dmi_interfacial(self, D):
        return lib().orc_add_dmi_interfacial(self.h, _ptr(self._vec(D, 1)))

    def add_anis(self, Ku, axis=(0, 0, 1)):
        return lib().orc_add_anis(self.h, _ptr(self._vec(Ku, 1)), *map(float, axis))

    def add_demag(self, Nx=0, Ny=0, Nz=0, tensor=None):
        t = None if tensor is None else np.ascontiguousarray(np.asarray(tensor, dtype=np.float64).reshape(-1))
        return lib().orc_add_demag(self.h, Nx, Ny, Nz, _ptr(t))

    def add_dmi_bulk_spatial(self, Dx, Dy, Dz):
        return lib().orc_add_dmi_bulk_spatial(self.h, _ptr(self._vec(Dx, 1)), _ptr(self._vec(Dy, 1)),
                                              _ptr(self._vec(Dz, 1)))

    def add_sot(self, aj, bj, p):
        return lib().orc_add_sot(self.h, _ptr(self._vec(aj, 1)), float(bj), *map(float, p))

    def add_stt_zhang_li(self, bJ, xi, ft=1.0):
        return lib().orc_add_stt_zhang_li(self.h, _ptr(self._vec(bJ, 3)), _ptr(self._vec(xi, 1)), float(ft))

    def add_stt_slonczewski(self, J, ft_beta, Lambda, P, xi, p):
        return lib().orc_add_stt_slonczewski(self.h, _ptr(self._vec(J, 1)), float(ft_beta), float(Lambda), float(P),
                                             float(xi), *map(float, p))

    def add_thermal_noise(self, T, T0=0.0, scaling=1.0, k_B=1.3806505e-23, seed=0, dt=1e-14):
        return lib().orc_add_thermal_noise(self.h, _ptr(self._vec(T, 1)), float(T0), float(scaling), float(k_B),
                                           int(seed), float(dt))

    def term_field(self, idx, m=None):
        f = np.zeros(3 * self.n)
        e = np.zeros(self.n)
        mm = None if m is None else np.ascontiguousarray(np.asarray(m, dtype=np.float64).reshape(-1))
        rc = lib().orc_term_field(self.h, idx, _ptr(mm), _ptr(f), _ptr(e))
        if rc != 0:
            raise IndexError(idx)
        return f, e

    def effective_field(self, m=None):
        f = np.zeros(3 * self.n)
        mm = None if m is None else np.ascontiguousarray(np.asarray(m, dtype=np.float64).reshape(-1))
        lib().orc_effective_field(self.h, _ptr(mm), _ptr(f))
        return f

    def llg_rhs(self, m=None):
        f = np.zeros(3 * self.n)
        mm = None if m is None else np.ascontiguousarray(np.asarray(m, dtype=np.float64).reshape(-1))
        lib().orc_llg_rhs(self.h, _ptr(mm), _ptr(f))
        return f

    def energy(self, nterms):
        per = np.zeros(max(nterms, 1))
        tot = lib().orc_energy(self.h, _ptr(per))
        return tot, per[:nterms]

    def rk4(self, dt, nsteps):
        lib().orc_rk4(self.h, float(dt), int(nsteps))

    def set_method(self, method):
        """0 DormandPrince, 1 BS23, 2 CashKarp54, 3 Fehlberg54."""
        lib().orc_set_method(self.h, int(method))

    def heun(self, dt, nsteps):
        lib().orc_heun(self.h, float(dt), int(nsteps))

    def rk4_time(self):
        return lib().orc_rk4_time(self.h)

    def set_tol(self, tol):
        lib().orc_dopri_set(self.h, float(tol))

    def run_until(self, t_end):
        st = np.zeros(6)
        ok = lib().orc_run_until(self.h, float(t_end), _ptr(st))
        return ok, dict(t=st[0], step=st[1], step_next=st[2], nsteps=int(st[3]), nfevals=int(st[4]), attempts=int(st[5]))

    def get_y_current(self):
        """The adaptive stepper's state (integrator.y_current)."""
        out = np.zeros(3 * self.n)
        lib().orc_get_y_current(self.h, _ptr(out))
        return out

    def dopri_advance(self):
        st = np.zeros(6)
        ok = lib().orc_dopri_advance(self.h, _ptr(st))
        return ok, dict(t=st[0], step=st[1], step_next=st[2], nsteps=int(st[3]), nfevals=int(st[4]), attempts=int(st[5]))

    def relax(self, driver="SD", max_steps=10000, stopping_dmdt=0.01):
        out = np.zeros(1)
        steps = lib().orc_relax(self.h, 0 if driver == "SD" else 1, int(max_steps), float(stopping_dmdt), _ptr(out))
        return int(steps), float(out[0])


def philox(counter, key):
    """Philox-4x32-10 of one 4-word counter block with a 2-word key."""
    c = (ctypes.c_uint32 * 4)(*counter)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().orc_philox(c, k, o)
    return list(o)
