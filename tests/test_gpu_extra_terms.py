"""The further terms on the GPU against the oracle: spatial bulk DMI
(SpatialVectorBulkDMI), SOT (add_sot), Zhang-Li and Slonczewski STT
(add_stt), thermal noise (add_thermal_noise), alone and together with the
base terms through RK4, Heun and Dormand-Prince stepping."""
import numpy as np
import pytest

from helpers import TERM_ID, GpuSim, build_oracle, extra_config, rel_maxnorm

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5
MESHES = [(9, 7, 3, ""), (8, 8, 1, "xy"), (5, 6, 4, "xyz")]
EXTRA = ("dmi_bulk_sp", "sot", "stt_zl", "stt_sl", "thermal")


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("mesh", MESHES)
@pytest.mark.parametrize("term", EXTRA)
def test_term_field_fp64(mesh, term):
    cfg = extra_config(11, *mesh, terms=(term,))
    o, idx = build_oracle(cfg)
    g = GpuSim(cfg, form=0)
    fo, eo = o.term_field(idx[term])
    fg, eg = g.term_field(term)
    assert rel_maxnorm(fg, fo) <= TOL64, term
    if term == "dmi_bulk_sp":
        assert rel_maxnorm(eg, eo) <= TOL64


def _all_cfg(mesh, T=None):
    cfg = extra_config(12, *mesh, terms=("exch", "dmi_int", "anis", "zeeman", "demag") + EXTRA)
    if T is not None:
        cfg["T"] = np.full(mesh[0] * mesh[1] * mesh[2], T)
        cfg["T0"] = 0.0
    return cfg


@pytest.mark.parametrize("mesh", MESHES)
def test_field_rhs_and_rk4_with_all_terms_fp64(mesh):
    from oracle.oracle import demag_tensor

    cfg = _all_cfg(mesh)
    T = demag_tensor(mesh[0], mesh[1], mesh[2], cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    assert rel_maxnorm(g.field(), o.effective_field()) <= TOL64
    assert rel_maxnorm(g.rhs(), o.llg_rhs()) <= TOL64
    o.rk4(2e-14, 1)
    g.rk4(2e-14, 1)
    assert rel_maxnorm(g.m(), o.get_m()) <= TOL64
    o.rk4(2e-14, 9)  # a new thermal draw every step
    g.rk4(2e-14, 9)
    assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11
    assert rel_maxnorm(g.field(), o.effective_field()) <= 1e-11  # draw of the step counter after 10 steps


def test_heun_and_dopri_with_all_terms_fp64():
    from oracle.oracle import demag_tensor

    mesh = (9, 7, 3, "")
    cfg = _all_cfg(mesh)
    T = demag_tensor(9, 7, 3, cfg["dx"], cfg["dy"], cfg["dz"])
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    o.heun(1e-14, 10)
    g.heun(1e-14, 10)
    assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11
    cfg = _all_cfg(mesh, T=1.0)  # a cold bath keeps the adaptive steps long enough
    o, _ = build_oracle(cfg, tensor=T)
    g = GpuSim(cfg, form=0, tensor=T)
    o.set_tol(1e-6)
    g.set_tol(1e-6)
    ok, so = o.run_until(1e-13)
    rc, sg = g.run_until(1e-13)
    assert ok and rc == 0
    assert sg["nsteps"] == so["nsteps"] and sg["nfevals"] == so["nfevals"]
    assert rel_maxnorm(g.m(), o.get_m()) <= 1e-11


@pytest.mark.parametrize("mesh", MESHES)
def test_fp32_form_fields_with_all_terms(mesh):
    cfg = _all_cfg(mesh)
    g64 = GpuSim(cfg, form=0)
    g32 = GpuSim(cfg, form=1)
    assert rel_maxnorm(g32.field(), g64.field()) <= TOL32
    assert rel_maxnorm(g32.rhs(), g64.rhs()) <= TOL32


@pytest.mark.parametrize("precision", [np.float32, np.float64])
def test_df_torque_api(precision):
    """test_df_torque  test/test_sot.jl:8-48 through the Python API."""
    import mmcuda as mm

    mm.set_precision(precision)
    try:
        mesh = mm.FDMesh(nx=1, ny=1, nz=1, dx=1e-9, dy=1e-9, dz=1e-9)
        sim = mm.Sim(mesh, name="spin", save_data=False)
    finally:
        mm.set_precision(np.float64)
    mm.set_Ms(sim, 8e5)
    sim.driver.alpha = 0.05
    sim.driver.gamma = 2.21e5
    sim.driver.integrator.tol = 1e-8
    mm.add_zeeman(sim, (0, 0, 1e5))
    aj, bj, p = 1e9, 5e8, (0.1, 0.2, 0.3)
    t = mm.add_sot(sim, aj, bj, p, name="dft_torque")
    mm.init_m0(sim, (-0.3, 0.4, 0.8), norm=False)
    m = np.array([-0.3, 0.4, 0.8])
    expected = (aj * np.cross(m, p) + bj * np.array(p)) / 2.21e5
    assert np.allclose(t.field, expected, rtol=1e-6)
    sim.close()


def test_adjoint_refuses_torque_terms():
    cfg = extra_config(13, 6, 5, 2, terms=("exch", "sot"))
    g = GpuSim(cfg, form=0)
    rc = g.L.mm_adjoint_record(g.h.h, 1e-14, 10, 5)
    assert rc == g.lib.MM_ERR_UNSUPPORTED if hasattr(g.lib, "MM_ERR_UNSUPPORTED") else rc == -7
