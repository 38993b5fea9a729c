"""The reference's own LLG tests (test/test_llg.jl) written against the Python
mirror of its API, run on the GPU in both precisions as the reference's
test_functions does (test/test_utils.jl:3-30)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def analytical(alpha, gamma, H0, t):
    """test/test_llg.jl:13-21."""
    p = gamma / (1 + alpha * alpha)
    beta = p * H0 * t
    return np.cos(beta) / np.cosh(alpha * beta), np.sin(beta) / np.cosh(alpha * beta), np.tanh(alpha * beta)


@pytest.fixture(params=[np.float32, np.float64], ids=["Float32", "Float64"])
def api(request):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mmcuda

    mmcuda.set_precision(request.param)
    yield mmcuda
    mmcuda.set_precision(np.float64)


@pytest.mark.parametrize("integrator", ["DormandPrince", "BS23", "CashKarp54", "Fehlberg54"])
def test_llg(api, integrator):
    """test_llg(integrator)  test/test_llg.jl:23-56."""
    tol = 1e-7 if integrator == "BS23" else 1e-8
    error = 2e-6 if integrator == "BS23" else 8e-7
    mesh = api.FDMesh(nx=1, ny=1, dx=1e-9)
    sim = api.Sim(mesh, name="spin", integrator=integrator, save_data=False)
    api.set_Ms(sim, 8e5)
    sim.driver.gamma = 2.21e5
    sim.driver.alpha = 0.05
    sim.driver.integrator.tol = tol
    api.add_zeeman(sim, (0, 0, 1e5))
    api.init_m0(sim, (1.0, 0, 0))
    for i in range(1, 11):
        api.run_until(sim, 1e-10 * i)
    mx, my, mz = analytical(0.05, 2.21e5, 1e5, 1e-9)
    m = sim.spin
    assert abs(mx - m[0]) < error
    assert abs(my - m[1]) < error
    assert abs(mz - m[2]) < error
    sim.close()


@pytest.mark.parametrize("integrator", ["Heun", "RungeKutta"])
def test_llg_fixed(api, integrator):
    """test_llg_fixed(integrator)  test/test_llg.jl:58-90: 500 run_step calls of dt = 1e-13."""
    mesh = api.FDMesh(nx=1, ny=1, dx=1e-9)
    sim = api.Sim(mesh, name="spin", integrator=integrator, save_data=False)
    api.set_Ms(sim, 8e5)
    sim.driver.alpha = 0.05
    sim.driver.gamma = 2.21e5
    sim.driver.integrator.step = 1e-13
    api.add_exch(sim, 1.3e-11)
    api.add_zeeman(sim, (0, 0, 1e5))
    api.init_m0(sim, (1.0, 0, 0))
    for _ in range(500):
        api.run_step(sim, sim.driver)
    assert abs(sim.driver.integrator.t - 5e-11) < 1e-22
    assert sim.driver.integrator.nsteps == 500
    mx, my, mz = analytical(0.05, 2.21e5, 1e5, 5e-11)
    m = sim.spin
    assert abs(mx - m[0]) < 8e-6
    assert abs(my - m[1]) < 8e-6
    assert abs(mz - m[2]) < 8e-6
    sim.close()


@pytest.mark.parametrize("ovf_type", ["Float64", "Float32", "String"])
def test_ovf_sim(api, tmp_path, ovf_type):
    """init_saving / test_sim_reading  test/test_ovf.jl:8-29 on a device Sim."""
    m = np.array([0.6, 0.8, 0, 0.6, 0.8, 0])
    mesh = api.FDMesh(nx=2, ny=1, nz=1, dx=1e-9, dy=1e-9, dz=1e-9)
    sim = api.Sim(mesh, name="saving", save_data=False)
    api.set_Ms(sim, 8.0e5)
    api.init_m0(sim, m)
    f = str(tmp_path / ovf_type)
    api.save_ovf(sim, f, type=ovf_type)
    sim2 = api.Sim(mesh, name="reading", save_data=False)
    api.set_Ms(sim2, 8.0e5)
    api.read_ovf(sim2, f)
    assert np.allclose(sim2.spin, m, atol=1e-6)
    ovf = api.read_ovf(f)
    assert ovf.name == "saving" and len(ovf.data) == 6 and np.max(np.abs(ovf.data - m)) < 1e-6
    sim.close()
    sim2.close()


@pytest.mark.parametrize("form", [0, 1])
def test_float32_host_boundary(form):
    """mm_set_m_f32 / mm_get_m_f32: sim.spin as a Float32 array (the
    reference's set_precision(Float32)) crosses the ABI unchanged, gives the
    same field as the Float64 copy of the same values, and is NaN-checked."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mmcuda import _lib

    nx, ny, nz = 24, 20, 3
    n = nx * ny * nz
    rng = np.random.default_rng(41)
    m = rng.normal(size=(n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    m32 = m.astype(np.float32).reshape(-1)
    hs = []
    for f32_in in (True, False):
        h = _lib.Handle(nx, ny, nz, 2e-9, 2e-9, 2e-9, 0, form, 0)
        h.call("mm_set_Ms", None, 6e5)
        h.call("mm_add_exch", None, 1.3e-11, 1.3e-11, 1.3e-11)
        h.call("mm_add_demag", 0, 0, 0)
        h.set_m(m32 if f32_in else m32.astype(np.float64))
        hs.append(h)
    assert np.array_equal(hs[0].get_m(), m32.astype(np.float64))
    assert np.array_equal(hs[0].get_m(dtype=np.float32), m32)
    f = []
    for h in hs:
        out = np.empty(3 * n)
        h.call("mm_effective_field", _lib.dptr(out))
        f.append(out)
    assert np.array_equal(f[0], f[1])
    hs[1].set_m(m.reshape(-1))
    got = hs[1].get_m(dtype=np.float32)
    assert np.allclose(got, m.reshape(-1).astype(np.float32), rtol=2 ** -23, atol=0)
    bad = m32.copy()
    bad[7] = np.nan
    with pytest.raises(_lib.MMError):
        hs[0].set_m(bad)
    for h in hs:
        h.close()
