"""The oracle's restatement of the further terms (spatial bulk DMI, SOT,
Zhang-Li and Slonczewski torques, thermal noise), pinned on the CPU."""
import numpy as np
import pytest

from oracle.oracle import OracleSim, philox

MU0 = 4e-7 * np.pi


def test_philox_known_answers():
    """Published Philox-4x32-10 known-answer vectors (Random123 kat_vectors)."""
    assert philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_df_torque():
    """test_df_torque  test/test_sot.jl:8-48: H = (aj (m x p) + bj p) / gamma."""
    s = OracleSim(1, 1, 1, 1e-9, 1e-9, 1e-9)
    s.set_Ms(8e5)
    s.set_llg(0.05, 2.21e5)
    s.add_zeeman([0, 0, 1e5])
    aj, bj, p = 1e9, 5e8, (0.1, 0.2, 0.3)
    idx = s.add_sot(aj, bj, p)
    m = np.array([-0.3, 0.4, 0.8])  # init_m0(..., norm=false)
    f, _ = s.term_field(idx, m)
    exp = (aj * np.cross(m, p) + bj * np.array(p)) / 2.21e5
    np.testing.assert_allclose(f, exp, rtol=1e-12)


def _film(nx=7, ny=5, nz=3, pbc=""):
    s = OracleSim(nx, ny, nz, 2e-9, 2.5e-9, 3e-9, pbc)
    rng = np.random.default_rng(3)
    n = nx * ny * nz
    Ms = rng.uniform(4e5, 9e5, n)
    Ms[rng.random(n) < 0.15] = 0
    m = rng.normal(size=(n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    m[Ms == 0] = 0
    s.set_Ms(Ms)
    s.set_m(m.reshape(-1))
    s.set_llg(0.1, 2.211e5)
    return s, rng, n, m.reshape(-1)


@pytest.mark.parametrize("pbc", ["", "xyz"])
def test_spatial_bulk_dmi_with_equal_arrays_is_bulk_dmi(pbc):
    """Equal D in every cell: the harmonic means are D, so SpatialVectorBulkDMI
    reproduces BulkDMI (kernels.jl:306-344 vs 347-422)."""
    s1, _, n, m = _film(pbc=pbc)
    s2, _, _, _ = _film(pbc=pbc)
    i1 = s1.add_dmi_bulk(3e-3, 2e-3, 1e-3)
    i2 = s2.add_dmi_bulk_spatial(np.full(n, 3e-3), np.full(n, 2e-3), np.full(n, 1e-3))
    f1, e1 = s1.term_field(i1, m)
    f2, e2 = s2.term_field(i2, m)
    np.testing.assert_allclose(f2, f1, rtol=1e-13, atol=1e-9 * np.max(np.abs(f1)))
    np.testing.assert_allclose(e2, e1, rtol=1e-12, atol=1e-12 * np.max(np.abs(e1)))


def test_zhang_li_field_of_a_linear_state():
    """(u.nabla) m by central differences inside, one-sided at the open ends."""
    nx = 6
    s = OracleSim(nx, 1, 1, 2e-9, 2e-9, 2e-9)
    s.set_Ms(8e5)
    s.set_llg(0.1, 2.2e5)
    x = np.arange(nx)
    m = np.stack([np.cos(0.1 * x), np.sin(0.1 * x), np.zeros(nx)], axis=1)
    s.set_m(m.reshape(-1))
    u = 7.0
    idx = s.add_stt_zhang_li(np.tile([u, 0, 0], nx), np.full(nx, 0.2), ft=1.0)
    f, _ = s.term_field(idx, m.reshape(-1))
    g = np.zeros_like(m)
    g[1:-1] = (m[2:] - m[:-2]) / (2 * 2e-9)
    g[0] = (m[1] - m[0]) / 2e-9
    g[-1] = (m[-1] - m[-2]) / 2e-9
    fu = u * g / 2.2e5
    exp = np.cross(m, fu) + 0.2 * fu
    np.testing.assert_allclose(f.reshape(-1, 3), exp, rtol=1e-12, atol=1e-12 * np.max(np.abs(exp)))


def test_slonczewski_field():
    s = OracleSim(1, 1, 1, 1e-9, 1e-9, 1e-9)
    s.set_Ms(8e5)
    m = np.array([0.6, 0.0, 0.8])
    s.set_m(m)
    p, P, Lam, xi, J, ftb = np.array([0.0, 0.6, 0.8]), 0.4, 2.0, 0.1, 1e11, 3e-12
    idx = s.add_stt_slonczewski(J, ftb, Lam, P, xi, p)
    f, _ = s.term_field(idx, m)
    eps = P * Lam ** 2 / (Lam ** 2 + 1 + (Lam ** 2 - 1) * (m @ p))
    np.testing.assert_allclose(f, J * ftb * (eps * np.cross(m, p) + xi * p), rtol=1e-13)


def test_thermal_field_statistics():
    """eta = H / sqrt(2 alpha k_B T / (V gamma dt mu0Ms)) is N(0,1), independent
    between components, cells and steps."""
    nx, ny, nz = 64, 64, 4
    s = OracleSim(nx, ny, nz, 2e-9, 2e-9, 2e-9)
    n = nx * ny * nz
    Ms = 8e5
    s.set_Ms(Ms)
    s.set_m(np.tile([0.0, 0.0, 1.0], n))
    s.set_llg(0.1, 2.211e5)
    T, dt = 300.0, 1e-14
    idx = s.add_thermal_noise(T, seed=12345, dt=dt)
    scale = np.sqrt(2 * 0.1 * 1.3806505e-23 * T / (8e-27 * 2.211e5 * dt * MU0 * Ms))
    f, _ = s.term_field(idx)
    eta = f.reshape(-1, 3) / scale
    assert abs(eta.mean()) < 4 / np.sqrt(eta.size)
    assert abs(eta.var() - 1) < 4 * np.sqrt(2 / eta.size)
    c = np.corrcoef(eta.T)
    assert np.max(np.abs(c - np.eye(3))) < 4 / np.sqrt(n)
    s.heun(dt, 1)  # the next step draws a new field
    f2, _ = s.term_field(idx)
    assert abs(np.corrcoef(f, f2)[0, 1]) < 4 / np.sqrt(eta.size)
