"""FP64 GPU parity at the benchmark's own workloads: the meshes, parameters and
seeded inputs that bench.py times (c1, c2, c4, c5 and the c3 film set with its
batch), against the CPU oracle, through the C ABI.

The paths these sizes take are the timed ones: c2's row-major z tiles with
leftover kx columns, c5's column-major spectra at 2048 x 2048 x 32, films whose
7-smooth padding differs from the oracle's 2n (nx = 251 pads to 504 here, 502
there), the batch graph of uneven meshes.  The Newell tensor is the GPU's own
(double-double near field) against the oracle's binary128 one.

Tolerances (relative max-norm): H_eff, dm/dt and one RK4 step 1e-12; a few
RK4 steps 1e-11; one Dormand-Prince step (initial-step estimate, controller,
7 stages): same accepted count and step, state 1e-11; FP32 form vs FP64 form
fields 1e-5.
"""
import numpy as np
import pytest

import bench
from helpers import rel_maxnorm

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_STEPS = 1e-11
TOL32 = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _oracle(w, m, H):
    """The oracle configured exactly as bench.setup_native configures the handle."""
    from oracle.oracle import OracleSim

    s = OracleSim(w["nx"], w["ny"], w["nz"], w["dx"], w["dy"], w["dz"])
    n = w["nx"] * w["ny"] * w["nz"]
    s.set_Ms(w["Ms"])
    s.set_m(m)
    s.set_llg(w["alpha"], w["gamma"])
    s.add_exch(Ax=w["A"], Ay=w["A"], Az=w["A"])
    if w["Dbulk"]:
        s.add_dmi_bulk(w["Dbulk"], w["Dbulk"], w["Dbulk"])
    if w["Ku"]:
        s.add_anis(np.full(n, w["Ku"]), w["axis"])
    if H is not None:
        s.add_zeeman(np.asarray(H))
    if w["demag"]:
        s.add_demag()
    return s


def _field(h):
    from mmcuda import _lib

    f = np.empty(3 * h.n)
    h.call("mm_effective_field", _lib.dptr(f))
    return f


def _rhs(h):
    from mmcuda import _lib

    f = np.empty(3 * h.n)
    h.call("mm_llg_rhs", _lib.dptr(f))
    return f


def _check_workload(wname, steps=(1,), form32=True):
    from mmcuda import _lib

    w = bench.WORKLOADS[wname]
    h, m0 = bench.setup_native(w, _lib.MM_FP64, 0)
    m, H = bench.synth_inputs(w)
    o = _oracle(w, m, H)
    ho = o.effective_field()
    assert rel_maxnorm(_field(h), ho) <= TOL64, (wname, "H_eff", rel_maxnorm(_field(h), ho))
    assert rel_maxnorm(_rhs(h), o.llg_rhs()) <= TOL64, (wname, "dm/dt")
    if form32:
        h32, _ = bench.setup_native(w, _lib.MM_FP32, 0)
        assert rel_maxnorm(_field(h32), ho) <= TOL32, (wname, "FP32 H_eff")
        h32.close()
    done = 0
    for k in steps:
        o.rk4(w["dt"], k - done)
        h.call("mm_rk4_run", w["dt"], k - done)
        done = k
        tol = TOL64 if k == 1 else TOL_STEPS
        err = rel_maxnorm(h.get_m(), o.get_m())
        assert err <= tol, (wname, k, "RK4 steps", err)
    h.close()
    return w, m0


def test_c1_film_inplane_zeeman():
    """200x50x1, 2.5x2.5x3 nm (non-cubic cell), exchange, demag, uniform
    in-plane Zeeman |B| <= 30 mT, alpha 0.02, RK4 dt = 1e-13."""
    _check_workload("c1", steps=(1, 5))


def test_c2_bulk_rk4():
    """256x256x64: exchange, bulk DMI, anisotropy, demag (row-major z tiles
    with leftover kx columns)."""
    _check_workload("c2", steps=(1,))


def test_c2_dormand_prince_step():
    """One Dormand-Prince step of c2 (tol 1e-6): initial-step estimate,
    controller on the device, error norm in FP64."""
    import ctypes

    from mmcuda import _lib

    w = bench.WORKLOADS["c2"]
    h, m0 = bench.setup_native(w, _lib.MM_FP64, 0)
    m, H = bench.synth_inputs(w)
    o = _oracle(w, m, H)
    o.set_tol(1e-6)
    h.call("mm_dopri_set_tol", 1e-6)
    ok, so = o.dopri_advance()
    st = _lib.Stats()
    _lib.check(_lib.load().mm_advance_step(h.h, ctypes.byref(st)))
    sg = st.asdict()
    assert ok and sg["nsteps"] == so["nsteps"] == 1
    assert abs(sg["step"] - so["step"]) <= 1e-12 * so["step"]
    assert abs(sg["t"] - so["t"]) <= 1e-12 * so["t"]
    # advance_step leaves sim.spin alone (adaptive_rk.jl:93-148): the state is
    # the integrator's y_current
    assert rel_maxnorm(h.get_m(), o.get_y_current()) <= TOL_STEPS
    h.close()


def test_c4_adjoint_mesh_fields():
    """128x128x4 of the adjoint workload: per-cell Ms ~ U[6,9]e5, exchange,
    interfacial DMI, anisotropy, demag; H_eff, dm/dt and one RK4 step."""
    from mmcuda import _lib
    from oracle.oracle import OracleSim

    w = bench.ADJOINT["c4"]
    n = w["nx"] * w["ny"] * w["nz"]
    rng = np.random.default_rng(w["seed"])
    m0 = rng.standard_normal((n, 3))
    m0 /= np.linalg.norm(m0, axis=1, keepdims=True)
    Ms = rng.uniform(6e5, 9e5, n)
    d = w["dx"]
    h = _lib.Handle(w["nx"], w["ny"], w["nz"], d, d, d, 0, _lib.MM_FP64)
    h.call("mm_set_Ms", _lib.dptr(Ms), 0.0)
    h.set_m(m0.reshape(-1))
    h.call("mm_set_llg", w["alpha"], w["gamma"], 1)
    h.call("mm_add_exch", None, w["A"], w["A"], w["A"])
    h.call("mm_add_dmi_interfacial", None, w["D"])
    h.call("mm_add_anis", None, w["Ku"], 0.0, 0.0, 1.0)
    h.call("mm_add_demag", 0, 0, 0)
    o = OracleSim(w["nx"], w["ny"], w["nz"], d, d, d)
    o.set_Ms(Ms)
    o.set_m(m0.reshape(-1))
    o.set_llg(w["alpha"], w["gamma"])
    o.add_exch(Ax=w["A"], Ay=w["A"], Az=w["A"])
    o.add_dmi_interfacial(np.full(n, w["D"]))
    o.add_anis(np.full(n, w["Ku"]), (0, 0, 1))
    o.add_demag()
    assert rel_maxnorm(_field(h), o.effective_field()) <= TOL64
    assert rel_maxnorm(_rhs(h), o.llg_rhs()) <= TOL64
    o.rk4(w["dt"], 1)
    h.call("mm_rk4_run", w["dt"], 1)
    assert rel_maxnorm(h.get_m(), o.get_m()) <= TOL64
    h.close()


def test_c5_column_major_full_size():
    """1024x1024x16 at 3 nm: column-major spectra of the padded
    2048x2048x32 grid at full size; H_eff, dm/dt and one RK4 step."""
    _check_workload("c5", steps=(1,), form32=True)


def _film_handle(s, form):
    from mmcuda import _lib

    h = _lib.Handle(s["nx"], s["ny"], s["nz"], 2e-9, 2e-9, 2e-9, 0, form)
    h.call("mm_set_Ms", None, s["Ms"])
    h.set_m(s["m"])
    h.call("mm_set_llg", 0.1, 2.211e5, 1)
    h.call("mm_add_exch", None, s["A"], s["A"], s["A"])
    h.call("mm_add_dmi_interfacial", None, s["D"])
    h.call("mm_add_demag", 0, 0, 0)
    return h


def _film_oracle(s):
    from oracle.oracle import OracleSim

    n = s["nx"] * s["ny"] * s["nz"]
    o = OracleSim(s["nx"], s["ny"], s["nz"], 2e-9, 2e-9, 2e-9)
    o.set_Ms(s["Ms"])
    o.set_m(s["m"])
    o.set_llg(0.1, 2.211e5)
    o.add_exch(Ax=s["A"], Ay=s["A"], Az=s["A"])
    o.add_dmi_interfacial(np.full(n, s["D"]))
    o.add_demag()
    return o


def test_c3_films_including_odd_padding():
    """Films of the c3 set plus nx = 251 (7-smooth padding 504 here, 502 in
    the oracle) and ny = 251: H_eff and one RK4 step each."""
    from mmcuda import _lib

    specs = bench.batch_specs("c3")
    rng = np.random.default_rng(251)
    extra = []
    for nx, ny, nz in ((251, 37, 2), (29, 251, 1), (251, 251, 3)):
        m = rng.standard_normal((nx * ny * nz, 3))
        m /= np.linalg.norm(m, axis=1, keepdims=True)
        extra.append(dict(nx=nx, ny=ny, nz=nz, D=2.5e-3, Ms=7e5, A=1.1e-11, m=m.reshape(-1)))
    for s in specs[:6] + extra:
        h = _film_handle(s, _lib.MM_FP64)
        o = _film_oracle(s)
        assert rel_maxnorm(_field(h), o.effective_field()) <= TOL64, (s["nx"], s["ny"], s["nz"])
        o.rk4(5e-14, 1)
        h.call("mm_rk4_run", 5e-14, 1)
        assert rel_maxnorm(h.get_m(), o.get_m()) <= TOL64, (s["nx"], s["ny"], s["nz"])
        h.close()


@pytest.mark.parametrize("wname", ["c3", "c3neb"])
def test_c3_batch_against_oracle(wname):
    """The whole batched workload (48 uneven films, or 32 NEB images of
    128x128x1) advanced by the batch graph, every mesh against its own oracle
    run: two RK4 steps of 5e-14 s."""
    from mmcuda import _lib

    specs = bench.batch_specs(wname)
    handles = [_film_handle(s, _lib.MM_FP64) for s in specs]
    b = _lib.Batch(handles)
    b.rk4_run(5e-14, 2)
    for s, h in zip(specs, handles):
        o = _film_oracle(s)
        o.rk4(5e-14, 2)
        err = rel_maxnorm(h.get_m(), o.get_m())
        assert err <= TOL_STEPS, (s["nx"], s["ny"], s["nz"], err)
    b.close()
    for h in handles:
        h.close()
