"""Shared builders for the parity tests: one seeded configuration instantiated
both on the CPU oracle and on libmmcuda (through the C ABI)."""
from __future__ import annotations

import ctypes
import math

import numpy as np

MU0 = 4 * math.pi * 1e-7


def rel_maxnorm(a, b):
    """||a - b||_inf / ||b||_inf (0 when both vanish)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.max(np.abs(a - b)) if a.size else 0.0
    s = np.max(np.abs(b)) if b.size else 0.0
    return 0.0 if d == 0 else d / max(s, 1e-300)


def random_config(seed, nx, ny, nz, pbc="", holes=True, terms=("exch", "dmi_bulk", "dmi_int", "anis", "zeeman", "demag"),
                  spatial=True, dx=2e-9, dy=2.5e-9, dz=3e-9):
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    Ms = rng.uniform(4e5, 9e5, n)
    if holes and n > 4:
        Ms[rng.random(n) < 0.15] = 0.0
    m = rng.normal(size=(n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    m[Ms == 0] = 0.0
    cfg = dict(nx=nx, ny=ny, nz=nz, dx=dx, dy=dy, dz=dz, pbc=pbc, Ms=Ms, m=m.reshape(-1), terms=list(terms))
    cfg["A"] = rng.uniform(0.8e-11, 1.5e-11, n) if spatial else 1.3e-11
    if spatial and n > 4:
        cfg["A"][rng.random(n) < 0.1] = 0.0
    cfg["Dbulk"] = (3e-3, 2.5e-3, 1.5e-3)
    cfg["Dint"] = rng.uniform(1e-3, 4e-3, n) if spatial else np.full(n, 2e-3)
    cfg["Ku"] = rng.uniform(-3e4, 5e5, n) if spatial else np.full(n, 5e5)
    cfg["axis"] = (0.3, -0.2, 0.9)
    cfg["H"] = rng.uniform(-3e4, 3e4, 3 * n)
    cfg["alpha"], cfg["gamma"] = 0.05, 2.211e5
    return cfg


def build_oracle(cfg, tensor=None):
    from oracle.oracle import OracleSim

    s = OracleSim(cfg["nx"], cfg["ny"], cfg["nz"], cfg["dx"], cfg["dy"], cfg["dz"], cfg["pbc"])
    s.set_Ms(cfg["Ms"])
    s.set_m(cfg["m"])
    s.set_llg(cfg["alpha"], cfg["gamma"])
    idx = {}
    n = s.n
    for t in cfg["terms"]:
        if t == "exch":
            A = cfg["A"]
            idx[t] = s.add_exch(A=A) if np.ndim(A) else s.add_exch(Ax=A, Ay=A, Az=A)
        elif t == "dmi_bulk":
            idx[t] = s.add_dmi_bulk(*cfg["Dbulk"])
        elif t == "dmi_int":
            idx[t] = s.add_dmi_interfacial(cfg["Dint"])
        elif t == "anis":
            idx[t] = s.add_anis(cfg["Ku"], cfg["axis"])
        elif t == "zeeman":
            idx[t] = s.add_zeeman(cfg["H"])
        elif t == "demag":
            idx[t] = s.add_demag(*cfg.get("macro", (0, 0, 0)), tensor=tensor)
        elif t == "dmi_bulk_sp":
            idx[t] = s.add_dmi_bulk_spatial(*cfg["bD"])
        elif t == "sot":
            idx[t] = s.add_sot(cfg["aj"], cfg["bj"], cfg["p"])
        elif t == "stt_zl":
            idx[t] = s.add_stt_zhang_li(cfg["bJ"], cfg["xi"], cfg["ft"])
        elif t == "stt_sl":
            idx[t] = s.add_stt_slonczewski(cfg["J"], cfg["ftb"], cfg["Lambda"], cfg["P"], cfg["xi_s"], cfg["p_sl"])
        elif t == "thermal":
            idx[t] = s.add_thermal_noise(cfg["T"], cfg["T0"], cfg["scaling"], seed=cfg["seed"], dt=cfg["th_dt"])
    assert len(idx) == len(cfg["terms"]) and n > 0
    return s, idx


def extra_config(seed, nx, ny, nz, pbc="", terms=("exch", "dmi_bulk_sp", "sot", "stt_zl", "stt_sl", "thermal")):
    """random_config plus the parameters of the further terms."""
    cfg = random_config(seed, nx, ny, nz, pbc, terms=terms)
    rng = np.random.default_rng(seed + 1000)
    n = nx * ny * nz
    cfg["bD"] = tuple(rng.uniform(1e-3, 4e-3, n) for _ in range(3))
    cfg["bD"][1][rng.random(n) < 0.1] = 0.0
    cfg["aj"] = rng.uniform(5e8, 2e9, n)
    cfg["bj"] = 3e8
    cfg["p"] = (0.1, 0.2, 0.3)
    cfg["bJ"] = rng.uniform(-50, 50, 3 * n)
    cfg["xi"] = rng.uniform(0.0, 0.2, n)
    cfg["ft"] = 0.7
    cfg["J"] = rng.uniform(5e10, 2e11, n)
    cfg["ftb"], cfg["Lambda"], cfg["P"], cfg["xi_s"], cfg["p_sl"] = 2.5e-12, 2.0, 0.4, 0.05, (0.0, 0.6, 0.8)
    cfg["T"] = rng.uniform(100, 400, n)
    cfg["T0"], cfg["scaling"], cfg["seed"], cfg["th_dt"] = 20.0, 0.8, 987654321, 2e-14
    return cfg


TERM_ID = {"zeeman": 0, "exch": 1, "dmi_bulk": 2, "dmi_int": 3, "anis": 4, "demag": 5, "dmi_bulk_sp": 2, "sot": 6,
           "stt_zl": 7, "stt_sl": 8, "thermal": 9}


class GpuSim:
    """Thin driver of one mm_handle for the parity tests (C ABI only)."""

    def __init__(self, cfg, form=0, tensor=None):
        from mmcuda import _lib

        self.L = _lib.load()
        self.lib = _lib
        self.cfg = cfg
        self.n = cfg["nx"] * cfg["ny"] * cfg["nz"]
        bits = (1 if "x" in cfg["pbc"] else 0) | (2 if "y" in cfg["pbc"] else 0) | (4 if "z" in cfg["pbc"] else 0)
        self.h = _lib.Handle(cfg["nx"], cfg["ny"], cfg["nz"], cfg["dx"], cfg["dy"], cfg["dz"], bits, form)
        c = self.h.call
        dp = _lib.dptr
        c("mm_set_Ms", dp(np.ascontiguousarray(cfg["Ms"], dtype=np.float64)), 0.0)
        self.h.set_m(cfg["m"])
        c("mm_set_llg", cfg["alpha"], cfg["gamma"], 1)
        for t in cfg["terms"]:
            if t == "exch":
                A = cfg["A"]
                if np.ndim(A):
                    c("mm_add_exch", dp(np.ascontiguousarray(A, dtype=np.float64)), 0.0, 0.0, 0.0)
                else:
                    c("mm_add_exch", None, A, A, A)
            elif t == "dmi_bulk":
                c("mm_add_dmi_bulk", *cfg["Dbulk"])
            elif t == "dmi_int":
                c("mm_add_dmi_interfacial", dp(np.ascontiguousarray(cfg["Dint"], dtype=np.float64)), 0.0)
            elif t == "anis":
                c("mm_add_anis", dp(np.ascontiguousarray(cfg["Ku"], dtype=np.float64)), 0.0, *cfg["axis"])
            elif t == "zeeman":
                c("mm_add_zeeman", dp(np.ascontiguousarray(cfg["H"], dtype=np.float64)), 0.0, 0.0, 0.0)
            elif t == "demag":
                if tensor is not None:
                    c("mm_add_demag_tensor", dp(np.ascontiguousarray(tensor, dtype=np.float64).reshape(-1)))
                else:
                    c("mm_add_demag", *cfg.get("macro", (0, 0, 0)))
            elif t == "dmi_bulk_sp":
                c("mm_add_dmi_bulk_spatial", *(dp(np.ascontiguousarray(x, dtype=np.float64)) for x in cfg["bD"]))
            elif t == "sot":
                c("mm_add_sot", dp(np.ascontiguousarray(cfg["aj"], dtype=np.float64)), 0.0, cfg["bj"], *cfg["p"])
            elif t == "stt_zl":
                c("mm_add_stt_zhang_li", dp(np.ascontiguousarray(cfg["bJ"], dtype=np.float64)),
                  dp(np.ascontiguousarray(cfg["xi"], dtype=np.float64)), 0.0, cfg["ft"])
            elif t == "stt_sl":
                c("mm_add_stt_slonczewski", dp(np.ascontiguousarray(cfg["J"], dtype=np.float64)), 0.0, cfg["ftb"],
                  cfg["Lambda"], cfg["P"], cfg["xi_s"], *cfg["p_sl"])
            elif t == "thermal":
                c("mm_add_thermal_noise", dp(np.ascontiguousarray(cfg["T"], dtype=np.float64)), 0.0, cfg["T0"],
                  cfg["scaling"], 1.3806505e-23, cfg["seed"], cfg["th_dt"])

    def term_field(self, name):
        f = np.empty(3 * self.n)
        e = np.empty(self.n)
        self.h.call("mm_term_field", TERM_ID[name], self.lib.dptr(f), self.lib.dptr(e))
        return f, e

    def field(self):
        f = np.empty(3 * self.n)
        self.h.call("mm_effective_field", self.lib.dptr(f))
        return f

    def rhs(self):
        f = np.empty(3 * self.n)
        self.h.call("mm_llg_rhs", self.lib.dptr(f))
        return f

    def energy(self):
        per = np.zeros(6)
        tot = ctypes.c_double()
        self.h.call("mm_energy", self.lib.dptr(per), ctypes.byref(tot))
        return tot.value, per

    def rk4(self, dt, n):
        self.h.call("mm_rk4_run", dt, n)

    def heun(self, dt, n):
        self.h.call("mm_heun_run", dt, n)

    def m(self):
        return self.h.get_m()

    def run_until(self, t):
        st = self.lib.Stats()
        rc = self.L.mm_run_until(self.h.h, t, ctypes.byref(st))
        return rc, st.asdict()

    def set_tol(self, tol):
        self.h.call("mm_dopri_set_tol", tol)

    def set_method(self, method):
        self.h.call("mm_set_adaptive_method", method)
