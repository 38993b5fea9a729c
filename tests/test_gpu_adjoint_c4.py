"""The adjoint workload at full size: 128x128x4 cells at 2 nm, exchange
(A = 1.3e-11) + interfacial DMI (D = 3e-3) + uniaxial anisotropy (Ku = 4e5
along z) + demag, per-cell Ms ~ U[6,9]e5, seeded random m0, alpha = 0.1,
gamma = 2.211e5; loss sum |m_T - m_target|^2 after 2000 RK4 steps of 5e-14 s
with checkpoints every 100 steps.  Gradients with respect to m0 (through the
torch.autograd.Function wrapper), per-cell Ms and D are checked against
central finite differences with h = 1e-6 (relative for Ms and D) on 64
seeded entries: 32 m0 components, 31 Ms cells and the scalar D (its central
difference Richardson-extrapolated, see below)."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

NX, NY, NZ, DT, NSTEPS, CKPT = 128, 128, 4, 5e-14, 2000, 100
FD_TOL = 1e-4


def _problem(seed=104):
    rng = np.random.default_rng(seed)
    n = NX * NY * NZ
    m0 = rng.normal(size=(n, 3))
    m0 /= np.linalg.norm(m0, axis=1, keepdims=True)
    target = rng.normal(size=(n, 3))
    target /= np.linalg.norm(target, axis=1, keepdims=True)
    return m0.reshape(-1), rng.uniform(6e5, 9e5, n), target.reshape(-1)


def _sim(mm, Ms, D=3e-3, precision=np.float64):
    mm.set_precision(precision)
    try:
        mesh = mm.FDMesh(nx=NX, ny=NY, nz=NZ, dx=2e-9, dy=2e-9, dz=2e-9)
        sim = mm.Sim(mesh, integrator="RungeKutta", name="c4", save_data=False)
    finally:
        mm.set_precision(np.float64)
    mm.set_Ms(sim, Ms)
    mm.add_exch(sim, 1.3e-11)
    mm.add_dmi(sim, D, type="interfacial")
    mm.add_anis(sim, 4e5, axis=(0, 0, 1))
    mm.add_demag(sim)
    sim.driver.alpha = 0.1
    sim.driver.gamma = 2.211e5
    sim.driver.integrator.step = DT
    return sim


def _loss(mm, m0, Ms, target, D=3e-3):
    sim = _sim(mm, Ms, D)
    sim.spin = m0
    mm.run_rk4(sim, NSTEPS)
    L = float(np.sum((sim.spin - target) ** 2))
    sim.close()
    return L


def test_c4_adjoint_vs_finite_differences():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mmcuda as mm
    from mmcuda.adjoint import RK4Function

    m0, Ms, target = _problem()
    sim = _sim(mm, Ms)
    x = torch.tensor(m0, dtype=torch.float64, requires_grad=True)
    mT = RK4Function.apply(x, sim, NSTEPS, DT, CKPT)
    loss = ((mT - torch.from_numpy(target)) ** 2).sum()
    loss.backward()
    g_m0 = x.grad.numpy()
    g_Ms, g_D = sim.adjoint_grads["Ms"], sim.adjoint_grads["D"].sum()
    assert abs(loss.item() - _loss(mm, m0, Ms, target)) <= 1e-12 * loss.item()
    sim.close()

    rng = np.random.default_rng(9)
    n = NX * NY * NZ
    ci = rng.choice(3 * n, 32, replace=False)
    cs = rng.choice(n, 31, replace=False)
    fd_m0, fd_Ms = [], []
    for i in ci:
        v = []
        for s in (1, -1):
            m = m0.copy()
            m[i] += s * 1e-6
            v.append(_loss(mm, m, Ms, target))
        fd_m0.append((v[0] - v[1]) / 2e-6)
    for i in cs:
        h = 1e-6 * Ms[i]
        v = []
        for s in (1, -1):
            M = Ms.copy()
            M[i] += s * h
            v.append(_loss(mm, m0, M, target))
        fd_Ms.append((v[0] - v[1]) / (2 * h))
    # D scales a term of every cell, so L(D) is strongly curved at this step:
    # the central difference with h = 1e-6 D is 1.8e-3 off (its error falls as
    # h^2: 1.8e-5 at 1e-7 D), so it is Richardson-extrapolated with h/2
    def cd(h):
        return (_loss(mm, m0, Ms, target, 3e-3 + h) - _loss(mm, m0, Ms, target, 3e-3 - h)) / (2 * h)

    hD = 1e-6 * 3e-3
    fd_D = (4 * cd(hD / 2) - cd(hD)) / 3
    e_m0 = np.max(np.abs(g_m0[ci] - fd_m0)) / np.max(np.abs(fd_m0))
    e_Ms = np.max(np.abs(g_Ms[cs] - fd_Ms)) / np.max(np.abs(fd_Ms))
    e_D = abs(g_D - fd_D) / abs(fd_D)
    print(f"c4 adjoint vs FD: m0 {e_m0:.2e}, Ms {e_Ms:.2e}, D {e_D:.2e} (dL/dD = {g_D:.6e})")
    assert e_m0 <= FD_TOL and e_Ms <= FD_TOL and e_D <= FD_TOL

    # the FP32 form's adjoint against the FP64 gradients just checked
    s32 = _sim(mm, Ms, precision=np.float32)
    s32.spin = m0
    L32, g32 = mm.rk4_grad(s32, lambda mT: (np.sum((mT - target) ** 2), 2 * (mT - target)), NSTEPS, DT, CKPT)
    s32.close()
    r_m0 = np.max(np.abs(g32["m0"] - g_m0)) / np.max(np.abs(g_m0))
    r_Ms = np.max(np.abs(g32["Ms"] - g_Ms)) / np.max(np.abs(g_Ms))
    print(f"c4 FP32 vs FP64 adjoint: m0 {r_m0:.2e}, Ms {r_Ms:.2e}, D {abs(g32['D'].sum() - g_D) / abs(g_D):.2e}")
