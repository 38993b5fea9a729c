"""GPU parity: libmmcuda (through its C ABI) against the CPU oracle and the
reference's golden vectors.

Tolerances (relative max-norm ||gpu - ref||_inf / ||ref||_inf):
  * FP64 form, local terms, LLG right-hand side, RK4 / DOPRI steps: 1e-12
  * FP64 form, demag with the oracle's tensor uploaded (pure convolution): 1e-12
  * FP64 form, demag with the tensor assembled on the GPU: 1e-12 against the
    oracle's accurate tensor (both evaluate the cancelling Newell sums beyond
    FP64 -- double-double on the GPU, binary128 in the oracle -- so every entry
    rounds correctly; see TENSOR_TOL)
  * FP32 form against the FP64 form: 1e-5
"""
import json
import math
import os

import numpy as np
import pytest

from helpers import GpuSim, build_oracle, random_config, rel_maxnorm

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL64 = 1e-12
TENSOR_TOL = 1e-12  # GPU-assembled tensor vs the oracle's binary128 tensor
TOL32 = 1e-5

def _seed(mesh):
    return mesh[0] * 10000 + mesh[1] * 100 + mesh[2]


LOCAL = ("exch", "dmi_bulk", "dmi_int", "anis", "zeeman")

MESHES = [
    (7, 5, 3, ""), (20, 5, 3, ""), (16, 16, 1, "xy"), (12, 1, 1, ""), (1, 1, 1, ""), (3, 2, 1, ""),
    (5, 4, 6, "xyz"), (33, 7, 2, "x"), (2, 1, 1, ""), (9, 11, 4, "z"), (64, 48, 1, ""), (1, 6, 5, "y"),
]


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("mesh", MESHES)
def test_local_terms_fp64(mesh):
    nx, ny, nz, pbc = mesh
    cfg = random_config(_seed(mesh), nx, ny, nz, pbc, terms=LOCAL)
    o, idx = build_oracle(cfg)
    g = GpuSim(cfg, form=0)
    for t in LOCAL:
        fo, eo = o.term_field(idx[t])
        fg, eg = g.term_field(t)
        assert rel_maxnorm(fg, fo) <= TOL64, (t, rel_maxnorm(fg, fo))
        assert rel_maxnorm(eg, eo) <= TOL64, (t, "energy", rel_maxnorm(eg, eo))
    assert rel_maxnorm(g.field(), o.effective_field()) <= TOL64
    assert rel_maxnorm(g.rhs(), o.llg_rhs()) <= TOL64


@pytest.mark.parametrize("mesh", MESHES)
def test_demag_convolution_fp64(mesh):
    """FFT convolution alone: the oracle's real-space tensor is uploaded."""
    from oracle.oracle import demag_tensor

    nx, ny, nz, pbc = mesh
    cfg = random_config(7 + _seed(mesh), nx, ny, nz, "", terms=("demag",))
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, idx = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    fo, eo = o.term_field(idx["demag"])
    fg, eg = g.term_field("demag")
    assert rel_maxnorm(fg, fo) <= TOL64, rel_maxnorm(fg, fo)
    assert rel_maxnorm(eg, eo) <= TOL64


@pytest.mark.parametrize("mesh", MESHES)
def test_demag_newell_fp64(mesh):
    nx, ny, nz, pbc = mesh
    cfg = random_config(11 + _seed(mesh), nx, ny, nz, "", terms=("demag",))
    o, idx = build_oracle(cfg)
    g = GpuSim(cfg, form=0)
    fo, _ = o.term_field(idx["demag"])
    fg, _ = g.term_field("demag")
    assert rel_maxnorm(fg, fo) <= TENSOR_TOL, rel_maxnorm(fg, fo)


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("mesh", [(3000, 2, 1), (4, 1800, 1), (2, 3, 700), (6, 1100, 3), (7300, 2, 1),
                                  (2, 3700, 1), (2, 3700, 3), (7300, 2, 2)])
def test_demag_long_lines(mesh, form):
    """Padded lines beyond the multi-line tiles: one line per block (x/2 = 3000,
    y = 3600, z = 1400, y = 2200 with z = 6) and lines beyond one block, run as
    global-memory radix stages (x/2 = 7350, y = 7500, films and 3-D), FP64 to
    1e-12 with the oracle's tensor and with the GPU's, FP32 to 1e-5."""
    from oracle.oracle import demag_tensor

    nx, ny, nz = mesh
    cfg = random_config(17 + nx + ny + nz, nx, ny, nz, "", terms=("demag",))
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, idx = build_oracle(cfg, tensor=T)
    fo, _ = o.term_field(idx["demag"])
    fg, _ = GpuSim(cfg, form=form, tensor=T).term_field("demag")
    assert rel_maxnorm(fg, fo) <= (TOL64 if form == 0 else TOL32)
    if form == 0:
        fn, _ = GpuSim(cfg, form=0).term_field("demag")  # tensor assembled on the GPU
        assert rel_maxnorm(fn, fo) <= TENSOR_TOL


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("mesh", [(100, 80, 1), (40, 600, 1), (24, 1300, 1), (6, 2400, 1)])
def test_film_paths(mesh, form):
    """The film paths by column length (padded y = 160, 1200, 2600, 4800):
    the fused column-major y convolution within the tile budget or filling one
    block (FP64 y = 1200, FP32 y = 2600), and the global-memory y stages for
    columns that fit no block (FP64 y = 2600, both forms at y = 4800); field
    and two RK4 steps against the oracle."""
    from oracle.oracle import demag_tensor

    nx, ny, nz = mesh
    cfg = random_config(29 + nx + ny, nx, ny, nz, "", terms=("exch", "demag"), spatial=False)
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=form, tensor=T)
    tol = TOL64 if form == 0 else TOL32
    assert rel_maxnorm(g.field(), o.effective_field()) <= tol
    o.rk4(2e-14, 2)
    g.rk4(2e-14, 2)
    assert rel_maxnorm(g.m(), o.get_m()) <= (1e-11 if form == 0 else TOL32)


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("mesh", [(6, 210, 16), (6, 410, 16), (5, 130, 64)])
def test_column_major_3d(mesh, form):
    """3-D meshes whose y lines leave row tiles narrower than 8 columns keep
    the spectra column-major and tile the z convolution along ky (FP64 from
    padded y = 420, FP32 from y = 840; nz = 16 and 64 give power-of-two z):
    field and two RK4 steps against the oracle."""
    from oracle.oracle import demag_tensor

    nx, ny, nz = mesh
    cfg = random_config(31 + nx + ny + nz, nx, ny, nz, "", terms=("exch", "demag"), spatial=False)
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=form, tensor=T)
    tol = TOL64 if form == 0 else TOL32
    assert rel_maxnorm(g.field(), o.effective_field()) <= tol
    o.rk4(2e-14, 2)
    g.rk4(2e-14, 2)
    assert rel_maxnorm(g.m(), o.get_m()) <= (1e-11 if form == 0 else TOL32)


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("mesh", [(32, 12, 16), (64, 10, 16)])
def test_zconv_leftover_columns(mesh, form):
    """Power-of-two nx gives Hx = nx + 1 spectrum columns (33, 65): the fused z
    convolution tiles all but the last along kx and the last along ky in the
    same launch; field against the oracle."""
    from oracle.oracle import demag_tensor

    nx, ny, nz = mesh
    cfg = random_config(37 + nx + ny, nx, ny, nz, "", terms=("demag",))
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, idx = build_oracle(cfg, tensor=T)
    fo, _ = o.term_field(idx["demag"])
    fg, _ = GpuSim(cfg, form=form, tensor=T).term_field("demag")
    assert rel_maxnorm(fg, fo) <= (TOL64 if form == 0 else TOL32)


def test_long_lines_rk4_and_dopri_fp64():
    """Stepping through the global-memory line stages, gated in the adaptive
    stepper's graph (y = 7500 film with exchange, anisotropy and Zeeman)."""
    from oracle.oracle import demag_tensor

    cfg = random_config(23, 2, 3700, 1, "", terms=("exch", "anis", "zeeman", "demag"), spatial=False)
    T = demag_tensor(2, 3700, 1, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    o.rk4(2e-14, 3)
    g.rk4(2e-14, 3)
    assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11
    o, _ = build_oracle(cfg, tensor=T)  # a fresh Sim for the adaptive stepper (its y_current is m0)
    g = GpuSim(cfg, form=0, tensor=T)
    o.set_tol(1e-6)
    g.set_tol(1e-6)
    ok, so = o.run_until(1e-13)
    rc, sg = g.run_until(1e-13)
    assert ok and rc == 0 and sg["nsteps"] == so["nsteps"]
    assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11


def test_demag_macro_pbc_fp64():
    cfg = random_config(5, 6, 5, 1, "", terms=("demag",))
    cfg["macro"] = (3, 2, 0)
    o, idx = build_oracle(cfg)
    g = GpuSim(cfg, form=0)
    assert rel_maxnorm(g.term_field("demag")[0], o.term_field(idx["demag"])[0]) <= TENSOR_TOL


def test_golden_fields_gpu():
    """test/test_fields.jl:25-59 at the reference tolerances, on the GPU."""
    gd = dict(np.load(os.path.join(GOLD, "fields_20x5x3.npz")))
    n = 300
    m = gd["m0"].reshape(-1, 3).copy()
    m[gd["Ms"] == 0] = 0
    cfg = dict(nx=20, ny=5, nz=3, dx=2.5e-9, dy=2.5e-9, dz=3e-9, pbc="", Ms=gd["Ms"], m=m.reshape(-1),
               terms=["exch", "demag", "dmi_bulk", "dmi_int", "anis"], A=1.3e-11, Dbulk=(4e-3, 4e-3, 4e-3),
               Dint=np.full(n, 2e-3), Ku=np.full(n, -3e4), axis=(0, 0, 1), H=np.zeros(3 * n), alpha=0.1,
               gamma=2.21e5)
    g = GpuSim(cfg, form=0)
    keys = {"exch": "exch", "demag": "demag", "dmi_bulk": "dmi", "dmi_int": "dmi_interfacial", "anis": "anis"}
    energies = {}
    for t, k in keys.items():
        f, e = g.term_field(t)
        assert np.max(np.abs(f - gd[k])) < 1e-5, (t, np.max(np.abs(f - gd[k])))
        energies[k] = e.sum()
    E = gd["energy"]
    assert abs((energies["demag"] - E[0]) / E[0]) < 1e-11
    for i, k in enumerate(["exch", "dmi", "dmi_interfacial", "anis"], start=1):
        assert abs((energies[k] - E[i]) / E[i]) < 1e-13, k


def test_demag_known_answers_gpu():
    cases = json.load(open(os.path.join(GOLD, "demag_known.json")))["cases"]
    for c in cases:
        n = c["nx"] * c["ny"] * c["nz"]
        mm = np.array(c["m"], float)
        mm /= np.linalg.norm(mm)
        cfg = dict(nx=c["nx"], ny=c["ny"], nz=c["nz"], dx=c["dx"], dy=c["dy"], dz=c["dz"], pbc="",
                   Ms=np.full(n, c["Ms"]), m=np.tile(mm, n), terms=["demag"], alpha=0.1, gamma=2.21e5)
        f = GpuSim(cfg, form=0).field()
        exp = np.array(c["field"])
        assert np.linalg.norm(f - exp) <= math.sqrt(np.finfo(float).eps) * np.linalg.norm(exp)


@pytest.mark.parametrize("mesh", [(20, 5, 3, ""), (16, 16, 1, "xy"), (9, 11, 4, "z")])
def test_rk4_steps_fp64(mesh):
    """One and ten RK4 steps (src/integrator/rk.jl:23-52) with all terms."""
    nx, ny, nz, pbc = mesh
    cfg = random_config(3, nx, ny, nz, pbc)
    from oracle.oracle import demag_tensor

    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    dt = 2e-14
    o.rk4(dt, 1)
    g.rk4(dt, 1)
    assert rel_maxnorm(g.m(), o.get_m()) <= TOL64
    o.rk4(dt, 9)
    g.rk4(dt, 9)
    assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11


def test_dopri_run_until_fp64():
    """run_until with Dormand-Prince: same accepted steps and state as the oracle."""
    from oracle.oracle import demag_tensor

    cfg = random_config(4, 12, 10, 2, "")
    T = demag_tensor(12, 10, 2, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    o.set_tol(1e-6)
    g.set_tol(1e-6)
    for t in (2e-13, 5e-13):
        ok, so = o.run_until(t)
        rc, sg = g.run_until(t)
        assert ok and rc == 0
        assert sg["nsteps"] == so["nsteps"] and sg["attempts"] - sg["rejected"] == so["nsteps"]
        assert abs(sg["t"] - so["t"]) <= 1e-15 * t
        assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11


@pytest.mark.parametrize("method", [1, 2, 3])
def test_adaptive_methods_run_until_fp64(method):
    """run_until with BS23 (FSAL), CashKarp54, Fehlberg54
    (src/integrator/adaptive_rk_steps.jl:11-229): same accepted steps,
    function evaluations and state as the oracle."""
    from oracle.oracle import demag_tensor

    cfg = random_config(40 + method, 12, 10, 2, "")
    T = demag_tensor(12, 10, 2, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    o.set_method(method)
    g.set_method(method)
    o.set_tol(1e-6)
    g.set_tol(1e-6)
    for t in (2e-13, 5e-13):
        ok, so = o.run_until(t)
        rc, sg = g.run_until(t)
        assert ok and rc == 0
        assert sg["nsteps"] == so["nsteps"] and sg["nfevals"] == so["nfevals"]
        assert abs(sg["t"] - so["t"]) <= 1e-15 * t
        assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11


@pytest.mark.parametrize("mesh", [(20, 5, 3, ""), (16, 16, 1, "xy"), (9, 11, 4, "z")])
def test_heun_steps_fp64(mesh):
    """One and ten Heun steps (src/integrator/heun.jl:28-49) with all terms."""
    nx, ny, nz, pbc = mesh
    cfg = random_config(5, nx, ny, nz, pbc)
    from oracle.oracle import demag_tensor

    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    dt = 1e-14
    o.heun(dt, 1)
    g.heun(dt, 1)
    assert rel_maxnorm(g.m(), o.get_m()) <= TOL64
    o.heun(dt, 9)
    g.heun(dt, 9)
    assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11


def analytical(alpha, gamma, H0, t):
    p = gamma / (1 + alpha * alpha)
    beta = p * H0 * t
    return np.cos(beta) / np.cosh(alpha * beta), np.sin(beta) / np.cosh(alpha * beta), np.tanh(alpha * beta)


@pytest.mark.parametrize("form", [0, 1])
def test_macrospin_rk4_and_dopri(form):
    """test/test_llg.jl:23-104 on the GPU: analytic damped precession."""
    cfg = dict(nx=1, ny=1, nz=1, dx=1e-9, dy=1e-9, dz=1e-9, pbc="", Ms=np.array([8e5]), m=np.array([1.0, 0, 0]),
               terms=["exch", "zeeman"], A=1.3e-11, H=np.array([0, 0, 1e5]), alpha=0.05, gamma=2.21e5)
    g = GpuSim(cfg, form=form)
    g.rk4(1e-13, 500)
    exp = analytical(0.05, 2.21e5, 1e5, 5e-11)
    m = g.m()
    assert all(abs(m[i] - exp[i]) < 8e-6 for i in range(3))
    cfg["terms"] = ["zeeman"]
    g = GpuSim(cfg, form=form)
    g.set_tol(1e-8)
    for i in range(1, 11):
        rc, _ = g.run_until(1e-10 * i)
        assert rc == 0
    exp = analytical(0.05, 2.21e5, 1e5, 1e-9)
    m = g.m()
    assert all(abs(m[i] - exp[i]) < 8e-7 for i in range(3))


@pytest.mark.parametrize("form", [0, 1])
def test_macrospin_heun_and_adaptive_methods(form):
    """test/test_llg.jl:23-120 on the GPU for Heun (dt 1e-13, 500 steps,
    |err| < 8e-6) and BS23 / CashKarp54 / Fehlberg54 (run_until 0.1..1 ns)."""
    cfg = dict(nx=1, ny=1, nz=1, dx=1e-9, dy=1e-9, dz=1e-9, pbc="", Ms=np.array([8e5]), m=np.array([1.0, 0, 0]),
               terms=["exch", "zeeman"], A=1.3e-11, H=np.array([0, 0, 1e5]), alpha=0.05, gamma=2.21e5)
    g = GpuSim(cfg, form=form)
    g.heun(1e-13, 500)
    exp = analytical(0.05, 2.21e5, 1e5, 5e-11)
    m = g.m()
    assert all(abs(m[i] - exp[i]) < 8e-6 for i in range(3))
    cfg["terms"] = ["zeeman"]
    exp = analytical(0.05, 2.21e5, 1e5, 1e-9)
    for method, tol, err in ((1, 1e-7, 2e-6), (2, 1e-8, 8e-7), (3, 1e-8, 8e-7)):
        g = GpuSim(cfg, form=form)
        g.set_method(method)
        g.set_tol(tol)
        for i in range(1, 11):
            rc, _ = g.run_until(1e-10 * i)
            assert rc == 0
        m = g.m()
        assert all(abs(m[i] - exp[i]) < err for i in range(3)), (method, m, exp)


def test_energies_fp64():
    from oracle.oracle import demag_tensor

    cfg = random_config(8, 10, 6, 3, "")
    T = demag_tensor(10, 6, 3, cfg["dx"], cfg["dy"], cfg["dz"])
    o, idx = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    tot, per = g.energy()
    for t, i in idx.items():
        eo = o.term_field(i)[1].sum()
        assert abs(per[{"zeeman": 0, "exch": 1, "dmi_bulk": 2, "dmi_int": 3, "anis": 4, "demag": 5}[t]] - eo) <= 1e-12 * abs(eo) + 1e-40


@pytest.mark.parametrize("driver", ["SD", "LLG"])
def test_relax_domain_wall_gpu(driver):
    """test/test_relax.jl:8-40 on the GPU, plus the step count of the oracle."""
    nx, ny, nz = 500, 1, 11
    n = nx * ny * nz
    m = np.zeros((nz, ny, nx, 3))
    i = np.arange(1, nx + 1)
    m[..., :] = np.where((i < 240)[:, None], [1, 0.1, 0], np.where((i < 260)[:, None], [0, 1, 0.1], [-1, 0.1, 0]))
    m /= np.linalg.norm(m, axis=-1, keepdims=True)
    cfg = dict(nx=nx, ny=ny, nz=nz, dx=2e-9, dy=2e-9, dz=1e-9, pbc="", Ms=np.full(n, 8.6e5), m=m.reshape(-1),
               terms=["exch", "anis"], A=1.3e-11, Ku=np.full(n, 1e5), axis=(1, 0, 0), alpha=0.5, gamma=2.21e5)
    g = GpuSim(cfg, form=0)
    o, _ = build_oracle(cfg)
    import ctypes

    if driver == "LLG":
        g.h.call("mm_set_llg", 0.5, 2.21e5, 0)
        o.set_llg(0.5, 2.21e5, precession=False)
    steps = ctypes.c_int64()
    mx = ctypes.c_double()
    g.h.call("mm_relax", 0 if driver == "SD" else 1, 2000, 0.1, ctypes.byref(steps), ctypes.byref(mx))
    so, _ = o.relax(driver, 2000, 0.1)
    mg = g.m().reshape(-1, 3).mean(0)
    assert abs(mg[0]) < 0.01 and abs(mg[1]) < 0.04 and abs(mg[2]) < 0.01
    assert abs(steps.value - so) <= max(2, so // 50), (steps.value, so)


@pytest.mark.parametrize("mesh", [(20, 5, 3, ""), (16, 16, 1, "xy"), (9, 11, 4, "z")])
def test_fp32_form_fields(mesh):
    nx, ny, nz, pbc = mesh
    cfg = random_config(9, nx, ny, nz, pbc)
    g64 = GpuSim(cfg, form=0)
    g32 = GpuSim(cfg, form=1)
    assert rel_maxnorm(g32.field(), g64.field()) <= TOL32
    assert rel_maxnorm(g32.rhs(), g64.rhs()) <= TOL32
    t64, p64 = g64.energy()
    t32, p32 = g32.energy()
    assert abs(t32 - t64) <= TOL32 * np.abs(p64).sum()


def smooth_film_cfg(nx=64, ny=32):
    """Film with exchange, in-plane Zeeman (30 mT) and demag started from a
    smooth non-uniform state: its dynamics are not chaotic (a 1e-10
    perturbation of the FP64 oracle stays ~1e-10 over 1000 steps while m
    rotates by O(1)), so FP32-vs-FP64 differences measure arithmetic error."""
    n = nx * ny
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    th = 0.4 * np.sin(2 * np.pi * X) + 0.2 * np.cos(2 * np.pi * Y)
    m = np.stack([np.cos(th), np.sin(th), 0.1 * np.sin(2 * np.pi * (X + Y))], -1).reshape(-1, 3)
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    H = np.tile([0.03 / (4e-7 * np.pi) * 0.8, 0.03 / (4e-7 * np.pi) * 0.6, 0.0], n)
    return dict(nx=nx, ny=ny, nz=1, dx=2.5e-9, dy=2.5e-9, dz=3e-9, pbc="", Ms=np.full(n, 8e5), m=m.reshape(-1),
                terms=["exch", "zeeman", "demag"], A=1.3e-11, H=H, alpha=0.02, gamma=2.211e5)


def test_fp32_form_rk4_1000_steps():
    """FP32 form vs FP64 form after 1000 RK4 steps (dt = 1e-13) on the smooth film."""
    cfg = smooth_film_cfg()
    g64 = GpuSim(cfg, form=0)
    g32 = GpuSim(cfg, form=1)
    g64.rk4(1e-13, 1000)
    g32.rk4(1e-13, 1000)
    err = rel_maxnorm(g32.m(), g64.m())
    print("fp32 vs fp64 after 1000 RK4 steps:", err)
    assert err <= TOL32


def test_fp32_form_rk4_random_state_short_horizon():
    """From random m the dynamics are chaotic (test_chaos_random_state in
    test_oracle_dynamics.py); over 50 steps FP32 stays within 1e-5 of FP64."""
    cfg = random_config(101, 64, 32, 1, "", holes=False, terms=("exch", "zeeman", "demag"), spatial=False)
    g64 = GpuSim(cfg, form=0)
    g32 = GpuSim(cfg, form=1)
    g64.rk4(1e-14, 50)
    g32.rk4(1e-14, 50)
    assert rel_maxnorm(g32.m(), g64.m()) <= TOL32


@pytest.mark.parametrize("mesh", [(128, 512, 16), (256, 1024, 16), (512, 512, 16), (1024, 512, 16), (256, 512, 64)])
def test_register_passes_fp32(mesh):
    """FP32 power-of-two meshes with ny >= 512 (nx = 128 .. 1024, nz = 16 or
    64) run the register-resident x and y passes (lane groups Q = 4 .. 32 for
    x, 16 and 32 for y) and, for nz = 16, the register-resident z convolution:
    the demag field, H_eff and two RK4 steps against the FP64 form of the same
    mesh (the FP64 form is pinned to the oracle by the other tests), and for
    the first mesh the two steps against the oracle too."""
    from oracle.oracle import demag_tensor

    nx, ny, nz = mesh
    cfg = random_config(41 + nx + ny + nz, nx, ny, nz, "", terms=("exch", "demag"), spatial=False)
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    g64 = GpuSim(cfg, form=0, tensor=T)
    g32 = GpuSim(cfg, form=1, tensor=T)
    assert rel_maxnorm(g32.term_field("demag")[0], g64.term_field("demag")[0]) <= TOL32
    assert rel_maxnorm(g32.field(), g64.field()) <= TOL32
    g32.rk4(2e-14, 2)
    g64.rk4(2e-14, 2)
    assert rel_maxnorm(g32.m(), g64.m()) <= TOL32
    if mesh == (128, 512, 16):
        o, _ = build_oracle(cfg, tensor=T)
        o.rk4(2e-14, 2)
        assert rel_maxnorm(g32.m(), o.get_m()) <= TOL32


@pytest.mark.parametrize("mesh", [(512, 1024, 2), (1024, 1024, 4)])
def test_register_passes_fp64(mesh):
    """FP64 meshes with nx = 512 or 1024 and ny = 1024 run the register-resident
    x passes (lane groups Q = 16, 32) and the bulk-copy y passes in FP64, with
    the shared-memory z convolution between them: H_eff and two RK4 steps
    against the oracle."""
    from oracle.oracle import demag_tensor

    nx, ny, nz = mesh
    cfg = random_config(47 + nx + nz, nx, ny, nz, "", terms=("exch", "demag"), spatial=False)
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    assert rel_maxnorm(g.field(), o.effective_field()) <= TOL64
    o.rk4(2e-14, 2)
    g.rk4(2e-14, 2)
    assert rel_maxnorm(g.m(), o.get_m()) <= TOL64


@pytest.mark.parametrize("mesh", [(64, 500, 16), (32, 1024, 16)])
def test_zquad_fp64(mesh):
    """FP64 column-major meshes with nz = 16 (Pz = 32) run the register z
    convolution of four threads a line: Py = 1000 (blocks past the last ky
    line, predicated) and Py = 2048 (every block full), the shared-memory x
    and y passes around it; H_eff and two RK4 steps against the oracle."""
    from oracle.oracle import demag_tensor

    nx, ny, nz = mesh
    cfg = random_config(53 + nx + ny, nx, ny, nz, "", terms=("exch", "dmi_bulk", "anis", "demag"), spatial=False)
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    assert rel_maxnorm(g.field(), o.effective_field()) <= TOL64
    o.rk4(2e-14, 2)
    g.rk4(2e-14, 2)
    assert rel_maxnorm(g.m(), o.get_m()) <= TOL64


def test_stage_tile_opt_in():
    """The halo-tiled stage kernel (MMCUDA_STAGETILE=1, off by default) gives
    the same RK4 steps as the default kernel: FP64 to 1e-12 against the
    oracle, in a process of its own (the switch is read once)."""
    import subprocess
    import sys

    code = (
        "import sys; sys.path[:0] = %r\n"
        "from helpers import GpuSim, build_oracle, random_config, rel_maxnorm\n"
        "for mesh in ((40, 24, 9, ''), (33, 17, 4, 'xyz'), (64, 1, 3, 'z')):\n"
        "    cfg = random_config(5 + mesh[0], *mesh)\n"
        "    o, _ = build_oracle(cfg)\n"
        "    g = GpuSim(cfg, form=0)\n"
        "    o.rk4(2e-14, 2); g.rk4(2e-14, 2)\n"
        "    e = rel_maxnorm(g.m(), o.get_m())\n"
        "    assert e <= 1e-11, (mesh, e)\n"
        "print('ok')\n" % ([ROOT, os.path.join(ROOT, "micromagnetic.jl_b200"), os.path.dirname(os.path.abspath(__file__))],))
    env = dict(os.environ, MMCUDA_STAGETILE="1")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


@pytest.mark.parametrize("mesh", [(100, 60, 16), (40, 900, 16)])
def test_zpair_layouts_fp32(mesh):
    """Pz = 32 (nz = 16) on meshes outside the register x / y passes: the
    register-resident z convolution on row-major spectra (100 x 60) and on
    column-major spectra (padded y = 1800): demag field against FP64."""
    from oracle.oracle import demag_tensor

    nx, ny, nz = mesh
    cfg = random_config(43 + nx + ny, nx, ny, nz, "", terms=("demag",))
    T = demag_tensor(nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    f64 = GpuSim(cfg, form=0, tensor=T).term_field("demag")[0]
    f32 = GpuSim(cfg, form=1, tensor=T).term_field("demag")[0]
    assert rel_maxnorm(f32, f64) <= TOL32
