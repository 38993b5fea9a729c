"""Host-side mirror of MicroMagnetic.jl's user API for the finite-difference
LLG path, driving libmmcuda.so.

Names, argument meanings, defaults and error behaviour follow the reference
(file:line citations below); Julia's keyword arguments become Python keyword
arguments and 1-based (i, j, k) callbacks stay 1-based.
"""
from __future__ import annotations

import math
import os
import warnings
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import Handle, check, dptr

mu_0 = 4 * math.pi * 1e-7  # src/const.jl:1
mu_B = 9.27400949e-24      # src/const.jl:2
k_B = 1.3806505e-23        # src/const.jl:3
c_e = 1.602176565e-19      # src/const.jl:4
h_bar = 1.05457172647e-34  # src/const.jl:9
mT = 0.001 / mu_0          # src/const.jl:13

_precision = [np.float64]  # global Float[] of src/MicroMagnetic.jl


def set_precision(t=np.float64):
    """set_precision(Float64 | Float32): form of the Sims created afterwards."""
    if t in (np.float64, float, "Float64", "double"):
        _precision[0] = np.float64
    elif t in (np.float32, "Float32", "float"):
        _precision[0] = np.float32
    else:
        raise ValueError("precision must be Float64 or Float32")


set_float = set_precision


def _form():
    return _lib.MM_FP32 if _precision[0] == np.float32 else _lib.MM_FP64


class FDMesh:
    """FDMesh(; dx, dy, dz, nx, ny, nz, pbc, x0, y0, z0)  src/micro/mesh.jl:69-98."""

    def __init__(self, dx=1e-9, dy=1e-9, dz=1e-9, nx=1, ny=1, nz=1, pbc="open", x0=None, y0=None, z0=None):
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.xperiodic = "x" in pbc
        self.yperiodic = "y" in pbc
        self.zperiodic = "z" in pbc
        self.n_total = self.nx * self.ny * self.nz
        self.volume = self.dx * self.dy * self.dz
        self.x0 = -self.nx * self.dx / 2 if x0 is None else x0
        self.y0 = -self.ny * self.dy / 2 if y0 is None else y0
        self.z0 = -self.nz * self.dz / 2 if z0 is None else z0

    @property
    def pbc_bits(self):
        return (1 if self.xperiodic else 0) | (2 if self.yperiodic else 0) | (4 if self.zperiodic else 0)


def _nargs(f):
    import inspect

    try:
        return len(inspect.signature(f).parameters)
    except (TypeError, ValueError):
        return 6


def _scalar_field(mesh: FDMesh, v) -> np.ndarray:
    """init_scalar!  src/helper.jl:5-45 (Number, Array, f(i,j,k,dx,dy,dz) or f(x,y,z))."""
    n = mesh.n_total
    if callable(v):
        out = np.zeros(n)
        na = _nargs(v)
        for k in range(1, mesh.nz + 1):
            for j in range(1, mesh.ny + 1):
                for i in range(1, mesh.nx + 1):
                    I = ((k - 1) * mesh.ny + (j - 1)) * mesh.nx + (i - 1)
                    if na == 3:
                        out[I] = v(mesh.x0 + (i - 0.5) * mesh.dx, mesh.y0 + (j - 0.5) * mesh.dy,
                                   mesh.z0 + (k - 0.5) * mesh.dz)
                    else:
                        out[I] = v(i, j, k, mesh.dx, mesh.dy, mesh.dz)
        return out
    a = np.asarray(v, dtype=np.float64)
    if a.ndim == 0:
        return np.full(n, float(a))
    a = a.reshape(-1)
    if a.size != n:
        raise ValueError(f"array of {a.size} entries for a mesh of {n} cells")
    return a.copy()


def _vector_field(mesh: FDMesh, v) -> np.ndarray:
    """init_vector!  src/helper.jl:47-104 (tuple, AoS array or f(i,j,k,dx,dy,dz) / f(x,y,z))."""
    n = mesh.n_total
    if callable(v):
        out = np.zeros((n, 3))
        na = _nargs(v)
        for k in range(1, mesh.nz + 1):
            for j in range(1, mesh.ny + 1):
                for i in range(1, mesh.nx + 1):
                    I = ((k - 1) * mesh.ny + (j - 1)) * mesh.nx + (i - 1)
                    if na == 3:
                        val = v((i - 0.5 - mesh.nx / 2) * mesh.dx, (j - 0.5 - mesh.ny / 2) * mesh.dy,
                                (k - 0.5 - mesh.nz / 2) * mesh.dz)
                    elif na == 6:
                        val = v(i, j, k, mesh.dx, mesh.dy, mesh.dz)
                    else:
                        raise ValueError("The input function should have either 6 or 3 arguments.")
                    if val is not None:
                        out[I] = val
        out = out.reshape(-1)
        if np.isnan(out).any():
            raise ValueError("NaN is given by the input function.")
        return out
    a = np.asarray(v, dtype=np.float64)
    if a.size == 3:
        return np.tile(a.reshape(3), n)
    a = a.reshape(-1)
    if a.size != 3 * n:
        raise ValueError(f"vector array of {a.size} entries for a mesh of {n} cells")
    return a.copy()


def _normalise(a: np.ndarray) -> None:
    """normalise  src/helper.jl:255-271."""
    v = a.reshape(-1, 3)
    m2 = np.einsum("ij,ij->i", v, v)
    ok = m2 > 0
    v[ok] /= np.sqrt(m2[ok])[:, None]


class Term:
    """An interaction term (src/head.jl:150-310).  `field` / `energy` are evaluated
    on access for the current magnetisation (the reference keeps the values of
    the last effective_field call)."""

    def __init__(self, sim, kind, name):
        self.sim, self.kind, self.name = sim, kind, name

    @property
    def field(self):
        f = np.empty(3 * self.sim.n_total)
        self.sim._h.call("mm_term_field", self.kind, dptr(f), None)
        return f

    @property
    def energy(self):
        e = np.empty(self.sim.n_total)
        self.sim._h.call("mm_term_field", self.kind, None, dptr(e))
        return e


# integrator name -> fixed-step entry point and default step, or adaptive
# method index (src/driver.jl:102-140)
_FIXED = {"RungeKutta": ("mm_rk4_run", 5e-14), "Heun": ("mm_heun_run", 1e-14)}
_INTEGRATORS = set(_FIXED) | set(_lib.RK_METHODS)


class _Integrator:
    def __init__(self, sim, name):
        self._sim = sim
        self.name = name
        self.adaptive = name in _lib.RK_METHODS
        self.kind = "AdaptiveRK" if self.adaptive else name
        self._step = 0.0 if self.adaptive else _FIXED[name][1]
        self._tol = 1e-6          # src/driver.jl:126
        if self.adaptive:
            sim._h.call("mm_set_adaptive_method", _lib.RK_METHODS[name])

    def run_fixed(self, nsteps, dt=None):
        """nsteps of the fixed-step scheme, one CUDA graph launch per step."""
        self._sim._h.call(_FIXED[self.name][0], float(self._step if dt is None else dt), int(nsteps))

    @property
    def step(self):
        if self.adaptive:
            return self._sim._stats().get("step", 0.0)
        return self._step

    @step.setter
    def step(self, v):
        self._step = float(v)

    @property
    def tol(self):
        return self._tol

    @tol.setter
    def tol(self, v):
        self._tol = float(v)
        self._sim._h.call("mm_dopri_set_tol", float(v))

    @property
    def t(self):
        if not self.adaptive:
            import ctypes

            t = ctypes.c_double()
            self._sim._h.call("mm_rk4_state", ctypes.byref(t), None)
            return t.value
        return self._sim._stats().get("t", 0.0)

    @property
    def nsteps(self):
        if not self.adaptive:
            import ctypes

            n = ctypes.c_int64()
            self._sim._h.call("mm_rk4_state", None, ctypes.byref(n))
            return n.value
        return self._sim._stats().get("nsteps", 0)


class _Driver:
    """LLG / SD driver parameters (src/driver.jl:3-21; defaults :95-102, :148)."""

    def __init__(self, sim, name, integrator):
        self._sim = sim
        self.name = name
        self._alpha, self._gamma, self._precession = 0.1, 2.21e5, True
        self.integrator = _Integrator(sim, integrator) if name == "LLG" else None

    def _push(self):
        self._sim._h.call("mm_set_llg", self._alpha, self._gamma, 1 if self._precession else 0)

    alpha = property(lambda s: s._alpha, lambda s, v: (setattr(s, "_alpha", float(v)), s._push()))
    gamma = property(lambda s: s._gamma, lambda s, v: (setattr(s, "_gamma", float(v)), s._push()))
    precession = property(lambda s: s._precession, lambda s, v: (setattr(s, "_precession", bool(v)), s._push()))


class Sim:
    """Sim(mesh; driver="LLG", name="dyn", integrator="DormandPrince", save_data=true)
    src/sim.jl:48-107 for an FDMesh; the state lives on `device`."""

    def __init__(self, mesh: FDMesh, driver="LLG", name="dyn", integrator="DormandPrince", save_data=True,
                 device=0):
        if driver not in ("LLG", "SD"):
            raise NotImplementedError(f"driver {driver!r} is outside the accelerated path (LLG, SD)")
        if driver == "LLG" and integrator not in _INTEGRATORS:
            raise NotImplementedError(
                f"integrator {integrator!r} is outside the accelerated path ({', '.join(sorted(_INTEGRATORS))})")
        self.mesh = mesh
        self.name = name
        self.n_total = mesh.n_total
        self.save_data = save_data
        self.device = device
        self.precision = _precision[0]
        self._h = Handle(mesh.nx, mesh.ny, mesh.nz, mesh.dx, mesh.dy, mesh.dz, mesh.pbc_bits, _form(), device)
        self.driver_name = driver
        self.driver = _Driver(self, driver, integrator)
        self.driver._push()
        self.interactions: list[Term] = []
        self._Ms = np.zeros(self.n_total)
        self._last_stats = {}
        self.saver_t = 0.0
        self.saver_nsteps = 0
        self._header_saved = False

    # -- state -------------------------------------------------------------
    @property
    def spin(self):
        return self._h.get_m()

    @spin.setter
    def spin(self, v):
        self._h.set_m(v)

    @property
    def mu0_Ms(self):
        return self._Ms * mu_0

    def _stats(self):
        return self._last_stats

    def close(self):
        self._h.close()


# -------------------------------------------------------------------- setup --
def set_Ms(sim: Sim, Ms):
    """set_Ms(sim, Ms)  src/sim.jl:129-143."""
    a = _scalar_field(sim.mesh, Ms)
    if np.isnan(a).any():
        raise ValueError("NaN is given by the input Ms!")
    sim._Ms = a
    sim._h.call("mm_set_Ms", dptr(np.ascontiguousarray(a)), 0.0)
    return True


def init_m0(sim: Sim, m0, norm=True):
    """init_m0(sim, m0; norm=true)  src/sim.jl:278-309."""
    spin = _vector_field(sim.mesh, m0)
    if norm:
        _normalise(spin)
    v = spin.reshape(-1, 3)
    v[sim._Ms == 0] = 0.0
    if np.isnan(spin).any():
        raise ValueError("NaN is given by the input m0!")
    sim._h.set_m(spin)
    return True


def set_pinning(sim: Sim, pins):
    """Pinned cells get dm/dt = 0 (llg.jl:14-19); pins: bool array or f(i,j,k,dx,dy,dz)."""
    a = _scalar_field(sim.mesh, pins).astype(np.uint8)
    import ctypes

    sim._h.call("mm_set_pins", a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))


def add_zeeman(sim: Sim, H0, ft=None, name="zeeman"):
    """add_zeeman(sim, H0; name)  src/micro/add_field.jl:11-48 (static field, A/m)."""
    if ft is not None:
        raise NotImplementedError("time-dependent Zeeman is outside the accelerated path")
    H = _vector_field(sim.mesh, H0)
    arr = np.asarray(H0).size != 3 or callable(H0)
    if arr:
        sim._h.call("mm_add_zeeman", dptr(np.ascontiguousarray(H)), 0.0, 0.0, 0.0)
    else:
        hx, hy, hz = (float(x) for x in np.asarray(H0, dtype=float).reshape(3))
        sim._h.call("mm_add_zeeman", None, hx, hy, hz)
    t = Term(sim, _lib.TERM_ZEEMAN, name)
    t.H0 = tuple(H0) if not arr else (0, 0, 0)
    sim.interactions.append(t)
    return t


def update_zeeman(sim: Sim, H0, name="zeeman"):
    """update_zeeman(sim, H0)  src/micro/add_field.jl:50-85 (replaces the static field)."""
    H = _vector_field(sim.mesh, H0)
    if np.asarray(H0).size != 3 or callable(H0):
        sim._h.call("mm_update_zeeman", dptr(np.ascontiguousarray(H)), 0.0, 0.0, 0.0)
    else:
        hx, hy, hz = (float(x) for x in np.asarray(H0, dtype=float).reshape(3))
        sim._h.call("mm_update_zeeman", None, hx, hy, hz)
    return True


def add_exch(sim: Sim, A, name="exch"):
    """add_exch(sim, A; name)  src/micro/add_field.jl:233-263."""
    if isinstance(A, (int, float, np.floating)):
        sim._h.call("mm_add_exch", None, float(A), float(A), float(A))
    elif isinstance(A, tuple) and len(A) == 3:
        sim._h.call("mm_add_exch", None, *(float(x) for x in A))
    else:
        a = _scalar_field(sim.mesh, A)
        sim._h.call("mm_add_exch", dptr(np.ascontiguousarray(a)), 0.0, 0.0, 0.0)
    t = Term(sim, _lib.TERM_EXCH, name)
    sim.interactions.append(t)
    return t


def add_dmi(sim: Sim, D, name="dmi", type="bulk"):
    """add_dmi(sim, D; name, type)  src/micro/add_field.jl:293-356."""
    if type == "bulk":
        if isinstance(D, (int, float, np.floating)):
            sim._h.call("mm_add_dmi_bulk", float(D), float(D), float(D))
            kind = _lib.TERM_DMI_BULK
        elif isinstance(D, tuple) and len(D) == 3 and all(isinstance(x, (int, float)) for x in D):
            sim._h.call("mm_add_dmi_bulk", *(float(x) for x in D))
            kind = _lib.TERM_DMI_BULK
        else:
            # SpatialVectorBulkDMI: a tuple of per-axis fields, or one field for all axes
            parts = D if (isinstance(D, tuple) and len(D) == 3) else (D, D, D)
            arrs = [np.ascontiguousarray(_scalar_field(sim.mesh, x)) for x in parts]
            sim._h.call("mm_add_dmi_bulk_spatial", *(dptr(a) for a in arrs))
            kind = _lib.TERM_DMI_BULK
    elif type == "interfacial":
        a = _scalar_field(sim.mesh, D)
        sim._h.call("mm_add_dmi_interfacial", dptr(np.ascontiguousarray(a)), 0.0)
        kind = _lib.TERM_DMI_INTERFACIAL
    elif type == "D2d":
        if not isinstance(D, (int, float, np.floating)):
            raise ValueError("D2d only support uniform DMI!")
        sim._h.call("mm_add_dmi_bulk", -float(D), float(D), 0.0)
        kind = _lib.TERM_DMI_BULK
    else:
        raise ValueError("Supported DMI type: interfacial bulk D2d")
    t = Term(sim, kind, name)
    sim.interactions.append(t)
    return t


def add_anis(sim: Sim, Ku, axis=(0, 0, 1), name="anis"):
    """add_anis(sim, Ku; axis, name)  src/micro/add_field.jl:430-465."""
    if callable(axis) or np.asarray(axis).size != 3:
        raise NotImplementedError("spatially varying anisotropy axes are outside the accelerated path")
    a = _scalar_field(sim.mesh, Ku)
    ax = [float(x) for x in axis]
    sim._h.call("mm_add_anis", dptr(np.ascontiguousarray(a)), 0.0, *ax)
    t = Term(sim, _lib.TERM_ANIS, name)
    sim.interactions.append(t)
    return t


def _const_scale(f, name):
    if callable(f):
        v = float(f(0.0))
        warnings.warn(f"{name}: a time-dependent scale is taken at t = 0 ({v}) on this path")
        return v
    return float(f)


def add_sot(sim: Sim, aj, bj, p, name="sot"):
    """add_sot(sim, aj, bj, p; name)  src/micro/add_field.jl:951-966:
    H = (aj/gamma) m x p + (bj/gamma) p."""
    a = _scalar_field(sim.mesh, aj)
    sim._h.call("mm_add_sot", dptr(np.ascontiguousarray(a)), 0.0, float(bj), *(float(x) for x in p))
    t = Term(sim, _lib.TERM_SOT, name)
    sim.interactions.append(t)
    return t


def add_stt(sim: Sim, model="slonczewski", **params):
    """add_stt(sim; model=:slonczewski | :zhang_li, kwargs...)  src/micro/add_field.jl:1134-1226."""
    model = str(model).lstrip(":")
    if "J" not in params:
        raise ValueError("Current density parameter `J` is required.")
    ft = _const_scale(params.get("ft", 1.0), "add_stt ft")
    if model == "zhang_li":
        has_b = "b" in params
        has_P = "P" in params and "Ms" in params
        if has_b:
            b = float(params["b"])
        elif has_P:
            b = params["P"] * mu_B / (c_e * params["Ms"])
        else:
            raise ValueError("Zhang-Li model requires either `b` or `(P, Ms)` parameters")
        xi = _scalar_field(sim.mesh, params.get("xi", 0.0))
        bJ = _vector_field(sim.mesh, params["J"]) * b
        if has_P and not has_b:
            bJ = (bJ.reshape(-1, 3) / (1 + xi ** 2)[:, None]).reshape(-1)
        sim._h.call("mm_add_stt_zhang_li", dptr(np.ascontiguousarray(bJ)), dptr(np.ascontiguousarray(xi)), 0.0, ft)
        t = Term(sim, _lib.TERM_STT_ZHANG_LI, params.get("name", "zhangli"))
    elif model == "slonczewski":
        for k in ("tf", "Ms", "p", "P"):
            if k not in params:
                raise ValueError(f"Parameter {k} is not provided")
        beta = h_bar / (mu_0 * params["Ms"] * c_e * params["tf"])
        J = _scalar_field(sim.mesh, params["J"])
        p = params["p"]
        sim._h.call("mm_add_stt_slonczewski", dptr(np.ascontiguousarray(J)), 0.0, ft * beta,
                    float(params.get("Lambda", 2.0)), float(params["P"]), float(params.get("xi", 0.0)),
                    *(float(x) for x in p))
        t = Term(sim, _lib.TERM_STT_SLONCZEWSKI, params.get("name", "slonczewski"))
    else:
        raise ValueError(f"Unsupported STT model: {model}. Supported models are: zhang_li, slonczewski")
    sim.interactions.append(t)
    return t


def add_thermal_noise(sim: Sim, Temp, name="thermal", T0=0.0, scaling=1.0, k_B=k_B, seed=0):
    """add_thermal_noise(sim, Temp; name, T0, scaling, k_B)  src/micro/add_field.jl:734-760.
    The noise of step n in cell i is a counter-based draw from `seed`."""
    if callable(Temp) and _nargs(Temp) == 4:
        raise NotImplementedError("space-time temperature profiles are outside the accelerated path")
    T = _scalar_field(sim.mesh, Temp)
    dt = float(sim.driver.integrator._step) if sim.driver.integrator is not None and sim.driver.integrator._step else 1e-14
    sim._h.call("mm_add_thermal_noise", dptr(np.ascontiguousarray(T)), 0.0, float(T0),
                _const_scale(scaling, "add_thermal_noise scaling"), float(k_B), int(seed), dt)
    t = Term(sim, _lib.TERM_THERMAL, name)
    sim.interactions.append(t)
    return t


def add_demag(sim: Sim, name="demag", Nx=0, Ny=0, Nz=0, fft=True):
    """add_demag(sim; name, Nx, Ny, Nz, fft)  src/micro/add_field.jl:403-419."""
    sim._h.call("mm_add_demag", int(Nx), int(Ny), int(Nz))
    t = Term(sim, _lib.TERM_DEMAG, name)
    sim.interactions.append(t)
    return t


# --------------------------------------------------------------- evaluation --
def effective_field(sim: Sim, spin=None, t: float = 0.0):
    """effective_field(sim, spin, t)  src/micro/field.jl:496-505; returns sim.field."""
    saved = None
    if spin is not None:
        saved = sim._h.get_m()
        sim._h.set_m(spin)
    try:
        out = np.empty(3 * sim.n_total)
        sim._h.call("mm_effective_field", dptr(out))
    finally:
        if saved is not None:
            sim._h.set_m(saved)
    sim.field = out
    return out


def compute_system_energy(sim: Sim, spin=None, t: float = 0.0):
    """compute_system_energy  src/micro/field.jl:520-536 -> total energy (J);
    per-term sums in sim.energies (FP64 device reductions)."""
    per = np.zeros(_lib.NTERMS)
    import ctypes

    tot = ctypes.c_double()
    sim._h.call("mm_energy", dptr(per), ctypes.byref(tot))
    sim.energies = per
    return tot.value


def average_m(sim: Sim):
    out = np.zeros(3)
    sim._h.call("mm_average_m", dptr(out))
    return out


def llg_rhs(sim: Sim):
    """dm/dt of llg_call_back (src/llg/llg.jl:45-59) at the current state."""
    out = np.empty(3 * sim.n_total)
    sim._h.call("mm_llg_rhs", dptr(out))
    return out


# -------------------------------------------------------------- integration --
def advance_step(sim: Sim):
    """advance_step(sim)  src/sim.jl:859-861 (one RK4 step or one adaptive step)."""
    integ = sim.driver.integrator
    if integ is None:
        raise ValueError("advance_step needs the LLG driver")
    if not integ.adaptive:
        integ.run_fixed(1)
        return True
    st = _lib.Stats()
    import ctypes

    rc = _lib.load().mm_advance_step(sim._h.h, ctypes.byref(st))
    sim._last_stats = st.asdict()
    if rc not in (0, -3, -4):
        check(rc)
    if rc != 0:
        warnings.warn(_lib.last_error())
    return rc == 0


def run_step(sim: Sim, driver=None):
    """run_step(sim, driver)  src/integrator/adaptive_rk.jl:269-271."""
    if sim.driver_name == "SD":
        steps = np.zeros(1)
        import ctypes

        n = ctypes.c_int64()
        check(_lib.load().mm_relax(sim._h.h, _lib.DRIVER_SD, 1, 0.0, ctypes.byref(n), dptr(steps)))
        return True
    return advance_step(sim)


def run_rk4(sim: Sim, nsteps: int, dt: float | None = None):
    """nsteps fixed RK4 steps (RungeKutta advance_step repeated, one graph launch each)."""
    integ = sim.driver.integrator
    if integ is None or integ.adaptive:
        raise ValueError("run_rk4 needs a fixed-step integrator (RungeKutta or Heun)")
    integ.run_fixed(nsteps, dt)


def run_until(sim: Sim, t_end: float, save_data=True):
    """run_until(sim, t_end; save_data)  src/sim.jl:547-579."""
    integ = sim.driver.integrator
    if integ is None or not integ.adaptive:
        raise ValueError("run_until needs an adaptive integrator (integrate_to_time is defined for AdaptiveRK only)")
    st = _lib.Stats()
    import ctypes

    rc = _lib.load().mm_run_until(sim._h.h, float(t_end), ctypes.byref(st))
    sim._last_stats = st.asdict()
    if rc not in (0, -3, -4):
        check(rc)
    if rc != 0:
        warnings.warn(f"Integration failed at t = {st.t}: {_lib.last_error()}")
    sim.saver_t = t_end
    if save_data and sim.save_data:
        write_data(sim)
    sim.saver_nsteps += 1
    return rc == 0


def run_sim(sim: Sim, steps=10, dt=1e-10, save_data=True, save_m_every=-1, call_back=None, **_):
    """run_sim(sim; steps, dt, save_data, save_m_every, call_back)  src/sim.jl:813-857."""
    if save_m_every is not None and save_m_every >= 0:
        warnings.warn("magnetisation snapshots (OVF) are not written on this path")
    for i in range(steps + 1):
        run_until(sim, i * dt, save_data=save_data)
        if call_back is not None:
            call_back(sim, i * dt)


def relax(sim: Sim, max_steps=10000, stopping_dmdt=0.01, save_data_every=0, save_m_every=0, **_):
    """relax(sim; max_steps, stopping_dmdt)  src/sim.jl:392-490 (SD or LLG driver)."""
    import ctypes

    drv = _lib.DRIVER_SD if sim.driver_name == "SD" else _lib.DRIVER_LLG
    n = ctypes.c_int64()
    mx = ctypes.c_double()
    check(_lib.load().mm_relax(sim._h.h, drv, int(max_steps), float(stopping_dmdt), ctypes.byref(n),
                               ctypes.byref(mx)))
    sim.relax_steps = n.value
    sim.max_dmdt = mx.value
    if save_data_every == 0 and sim.save_data:
        write_data(sim)
    return None


def set_driver(sim: Sim, driver="LLG", integrator="DormandPrince", **args):
    """set_driver(sim; driver, integrator, args...)  src/sim.jl:586-626 (alpha, gamma, precession)."""
    if driver not in ("LLG", "SD"):
        raise NotImplementedError(f"driver {driver!r} is outside the accelerated path")
    if driver == "LLG" and integrator not in _INTEGRATORS:
        raise NotImplementedError(f"integrator {integrator!r} is outside the accelerated path")
    if driver != sim.driver_name or (sim.driver.integrator and integrator != sim.driver.integrator.name):
        old = sim.driver
        sim.driver = _Driver(sim, driver, integrator)
        sim.driver._alpha, sim.driver._gamma, sim.driver._precession = old._alpha, old._gamma, old._precession
        sim.driver_name = driver
        sim._h.call("mm_dopri_reset")
    for k, v in args.items():
        if k in ("alpha", "gamma", "precession"):
            setattr(sim.driver, k, v)
        elif k in ("tol",) and sim.driver.integrator is not None:
            sim.driver.integrator.tol = v
        elif k in ("step", "dt") and sim.driver.integrator is not None:
            sim.driver.integrator.step = v
    sim.driver._push()


# --------------------------------------------------------------- saving ----
def write_data(sim: Sim):
    """DataSaver table  src/fileio.jl:73-97: step, time, E_total, <m>, E per term."""
    if not sim.save_data:
        return
    E = compute_system_energy(sim)
    m = average_m(sim)
    fname = f"{sim.name}_{sim.driver_name.lower()}.txt"
    names = [t.name for t in sim.interactions if t.kind < _lib.NTERMS]  # torque fields carry no energy
    if not sim._header_saved:
        with open(fname, "w") as f:
            cols = ["step", "time", "E_total", "m_x", "m_y", "m_z"] + [f"E_{n}" for n in names]
            f.write("#" + "".join(f"{c:>18s}" for c in cols) + "\n")
        sim._header_saved = True
    per = [sim.energies[t.kind] for t in sim.interactions if t.kind < _lib.NTERMS]
    with open(fname, "a") as f:
        vals = [sim.saver_nsteps, sim.saver_t, E, *m, *per]
        f.write(" " + "".join(f"{v:18.10e}" if isinstance(v, float) else f"{v:18d}" for v in vals) + "\n")
