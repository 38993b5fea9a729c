"""ctypes binding of libmmcuda.so (the C ABI declared in include/mmcuda.h).

The library is the product's only compute path: if it is missing or cannot
be loaded this module raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmmcuda.so")

MM_OK = 0
MM_ERR_ARG, MM_ERR_CUDA, MM_ERR_NAN, MM_ERR_NOCONVERGE = -1, -2, -3, -4
MM_ERR_TIMEOUT, MM_ERR_STATE, MM_ERR_UNSUPPORTED = -5, -6, -7
STATUS = {
    -1: "MM_ERR_ARG",
    -2: "MM_ERR_CUDA",
    -3: "MM_ERR_NAN",
    -4: "MM_ERR_NOCONVERGE",
    -5: "MM_ERR_TIMEOUT",
    -6: "MM_ERR_STATE",
    -7: "MM_ERR_UNSUPPORTED",
}
MM_FP64, MM_FP32 = 0, 1
MM_RK_DORMAND_PRINCE, MM_RK_BS23, MM_RK_CASH_KARP54, MM_RK_FEHLBERG54 = 0, 1, 2, 3
MM_OVF_TEXT, MM_OVF_BINARY4, MM_OVF_BINARY8 = 0, 4, 8
RK_METHODS = {"DormandPrince": 0, "DOPRI54": 0, "BS23": 1, "CashKarp54": 2, "Fehlberg54": 3, "RKF54": 3}
TERM_ZEEMAN, TERM_EXCH, TERM_DMI_BULK, TERM_DMI_INTERFACIAL, TERM_ANIS, TERM_DEMAG = range(6)
TERM_SOT, TERM_STT_ZHANG_LI, TERM_STT_SLONCZEWSKI, TERM_THERMAL = 6, 7, 8, 9
NTERMS = 6
DRIVER_SD, DRIVER_LLG = 0, 1

# every exported symbol of include/mmcuda.h
EXPORTS = (
    "mm_abi_version", "mm_last_error", "mm_create", "mm_destroy", "mm_get_stream", "mm_synchronize",
    "mm_device_bytes", "mm_set_Ms", "mm_set_m", "mm_get_m", "mm_set_m_f32", "mm_get_m_f32", "mm_set_pins", "mm_set_llg", "mm_add_zeeman",
    "mm_update_zeeman", "mm_add_exch", "mm_add_dmi_bulk", "mm_add_dmi_interfacial", "mm_add_anis",
    "mm_add_demag", "mm_add_demag_tensor", "mm_effective_field", "mm_term_field", "mm_energy",
    "mm_llg_rhs", "mm_average_m", "mm_rk4_run", "mm_rk4_state", "mm_dopri_set_tol", "mm_run_until",
    "mm_advance_step", "mm_dopri_reset", "mm_relax", "mm_kernel_time", "mm_rk4_launches_per_step",
    "mm_energy_noalloc", "mm_batch_create", "mm_batch_rk4_run", "mm_batch_get_stream", "mm_batch_launches", "mm_batch_destroy",
    "mm_heun_run", "mm_set_adaptive_method", "mm_ovf_write", "mm_ovf_read_header", "mm_ovf_read",
    "mm_save_ovf", "mm_load_ovf", "mm_adjoint_record", "mm_adjoint_backward", "mm_add_dmi_bulk_spatial",
    "mm_add_sot", "mm_add_stt_zhang_li", "mm_add_stt_slonczewski", "mm_add_thermal_noise", "mm_demag_tiles",
)
KERNELS = ("demag_fwd_x", "demag_fwd_y", "demag_conv", "demag_inv_y", "demag_inv_x", "rk4_stage", "rk4_step")


class MMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class MeshDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("pbc", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("step", ctypes.c_double), ("step_next", ctypes.c_double),
                ("nsteps", ctypes.c_int64), ("nfevals", ctypes.c_int64), ("attempts", ctypes.c_int64),
                ("rejected", ctypes.c_int64), ("status", ctypes.c_int32)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


def load():
    """Load libmmcuda.so (raises if it is absent: build it with build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libmmcuda.so not found at {LIB_PATH}; run micromagnetic.jl_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    i, d, i64 = ctypes.c_int, ctypes.c_double, ctypes.c_int64
    sig = {
        "mm_abi_version": ([], i),
        "mm_last_error": ([ctypes.c_char_p, ctypes.c_size_t], i),
        "mm_create": ([ctypes.POINTER(MeshDesc), i, i, ctypes.POINTER(_vp)], i),
        "mm_destroy": ([_vp], i),
        "mm_get_stream": ([_vp, ctypes.POINTER(_vp)], i),
        "mm_synchronize": ([_vp], i),
        "mm_device_bytes": ([_vp, ctypes.POINTER(ctypes.c_size_t)], i),
        "mm_set_Ms": ([_vp, _dp, d], i),
        "mm_set_m": ([_vp, _dp], i),
        "mm_get_m": ([_vp, _dp], i),
        "mm_set_m_f32": ([_vp, _fp], i),
        "mm_get_m_f32": ([_vp, _fp], i),
        "mm_set_pins": ([_vp, ctypes.POINTER(ctypes.c_uint8)], i),
        "mm_set_llg": ([_vp, d, d, i], i),
        "mm_add_zeeman": ([_vp, _dp, d, d, d], i),
        "mm_update_zeeman": ([_vp, _dp, d, d, d], i),
        "mm_add_exch": ([_vp, _dp, d, d, d], i),
        "mm_add_dmi_bulk": ([_vp, d, d, d], i),
        "mm_add_dmi_interfacial": ([_vp, _dp, d], i),
        "mm_add_anis": ([_vp, _dp, d, d, d, d], i),
        "mm_add_demag": ([_vp, i, i, i], i),
        "mm_add_demag_tensor": ([_vp, _dp], i),
        "mm_effective_field": ([_vp, _dp], i),
        "mm_term_field": ([_vp, i, _dp, _dp], i),
        "mm_energy": ([_vp, _dp, _dp], i),
        "mm_llg_rhs": ([_vp, _dp], i),
        "mm_average_m": ([_vp, _dp], i),
        "mm_rk4_run": ([_vp, d, i64], i),
        "mm_rk4_state": ([_vp, _dp, ctypes.POINTER(i64)], i),
        "mm_heun_run": ([_vp, d, i64], i),
        "mm_set_adaptive_method": ([_vp, i], i),
        "mm_ovf_write": ([ctypes.c_char_p, ctypes.POINTER(MeshDesc), _dp, i, ctypes.c_char_p], i),
        "mm_ovf_read_header": ([ctypes.c_char_p, ctypes.POINTER(MeshDesc), ctypes.POINTER(i), ctypes.c_char_p,
                                ctypes.c_size_t], i),
        "mm_ovf_read": ([ctypes.c_char_p, _dp, i64], i),
        "mm_save_ovf": ([_vp, ctypes.c_char_p, i, ctypes.c_char_p], i),
        "mm_load_ovf": ([_vp, ctypes.c_char_p], i),
        "mm_adjoint_record": ([_vp, d, i64, i64], i),
        "mm_add_dmi_bulk_spatial": ([_vp, _dp, _dp, _dp], i),
        "mm_demag_tiles": ([_vp, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_float)], i),
        "mm_add_sot": ([_vp, _dp, d, d, d, d, d], i),
        "mm_add_stt_zhang_li": ([_vp, _dp, _dp, d, d], i),
        "mm_add_stt_slonczewski": ([_vp, _dp, d, d, d, d, d, d, d, d], i),
        "mm_add_thermal_noise": ([_vp, _dp, d, d, d, d, ctypes.c_uint64, d], i),
        "mm_adjoint_backward": ([_vp, _dp, _dp, _dp, _dp, _dp], i),
        "mm_dopri_set_tol": ([_vp, d], i),
        "mm_run_until": ([_vp, d, ctypes.POINTER(Stats)], i),
        "mm_advance_step": ([_vp, ctypes.POINTER(Stats)], i),
        "mm_dopri_reset": ([_vp], i),
        "mm_relax": ([_vp, i, i64, d, ctypes.POINTER(i64), _dp], i),
        "mm_kernel_time": ([_vp, i, i, _dp, _dp], i),
        "mm_rk4_launches_per_step": ([_vp, ctypes.POINTER(i)], i),
        "mm_energy_noalloc": ([ctypes.POINTER(MeshDesc), _vp, _vp] + [d] * 9 + [_vp, _vp], i),
        "mm_batch_create": ([ctypes.POINTER(_vp), i, ctypes.POINTER(_vp)], i),
        "mm_batch_rk4_run": ([_vp, d, i64], i),
        "mm_batch_get_stream": ([_vp, ctypes.POINTER(_vp)], i),
        "mm_batch_launches": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], i),
        "mm_batch_destroy": ([_vp], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    load().mm_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != MM_OK:
        raise MMError(rc, last_error())


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


class Batch:
    """Owns one mm_batch over a list of Handles (kept alive by the batch)."""

    def __init__(self, handles):
        self.handles = list(handles)
        arr = (_vp * len(self.handles))(*[h.h for h in self.handles])
        self.b = _vp()
        check(load().mm_batch_create(arr, len(self.handles), ctypes.byref(self.b)))

    def rk4_run(self, dt, nsteps):
        check(load().mm_batch_rk4_run(self.b, float(dt), int(nsteps)))

    def stream(self) -> int:
        s = _vp()
        check(load().mm_batch_get_stream(self.b, ctypes.byref(s)))
        return int(s.value or 0)

    def launches(self):
        """(kernel launches of one batched RK4 step, handles in merged launches)."""
        n, k = ctypes.c_int(), ctypes.c_int()
        check(load().mm_batch_launches(self.b, ctypes.byref(n), ctypes.byref(k)))
        return n.value, k.value

    def close(self):
        if getattr(self, "b", None) and _lib is not None:
            _lib.mm_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        self.close()


class Handle:
    """Owns one mm_handle."""

    def __init__(self, nx, ny, nz, dx, dy, dz, pbc_bits, form, device=0):
        L = load()
        self.h = _vp()
        desc = MeshDesc(nx, ny, nz, dx, dy, dz, pbc_bits)
        check(L.mm_create(ctypes.byref(desc), form, device, ctypes.byref(self.h)))
        self.n = nx * ny * nz
        self.form = form

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.mm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def call(self, name, *args):
        check(getattr(load(), name)(self.h, *args))

    def stream(self) -> int:
        s = _vp()
        self.call("mm_get_stream", ctypes.byref(s))
        return int(s.value or 0)

    def device_bytes(self) -> int:
        b = ctypes.c_size_t()
        self.call("mm_device_bytes", ctypes.byref(b))
        return int(b.value)

    def kernel_time(self, kernel: int, reps: int = 20):
        """(ms per launch, algorithmic bytes per launch) of one library kernel."""
        ms, b = ctypes.c_double(), ctypes.c_double()
        self.call("mm_kernel_time", int(kernel), int(reps), ctypes.byref(ms), ctypes.byref(b))
        return ms.value, b.value

    def rk4_launches(self) -> int:
        n = ctypes.c_int()
        self.call("mm_rk4_launches_per_step", ctypes.byref(n))
        return n.value

    def get_m(self, out=None, dtype=np.float64):
        """m (AoS); dtype float32 copies out through mm_get_m_f32."""
        f32 = (out.dtype if out is not None else np.dtype(dtype)) == np.float32
        out = np.empty(3 * self.n, dtype=np.float32 if f32 else np.float64) if out is None else out
        if f32:
            self.call("mm_get_m_f32", fptr(out))
        else:
            self.call("mm_get_m", dptr(out))
        return out

    def set_m(self, m):
        """m (AoS); a float32 array is copied in through mm_set_m_f32."""
        f32 = isinstance(m, np.ndarray) and m.dtype == np.float32
        a = np.ascontiguousarray(m, dtype=np.float32 if f32 else np.float64).reshape(-1)
        if a.size != 3 * self.n:
            raise ValueError("m must have 3N entries")
        if f32:
            self.call("mm_set_m_f32", fptr(a))
        else:
            self.call("mm_set_m", dptr(a))
