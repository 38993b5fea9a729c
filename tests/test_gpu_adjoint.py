"""Reverse-mode gradients through fixed-step RK4 (mm_adjoint_record /
mm_adjoint_backward) against central finite differences of the forward
path, in the shape of the c4 workload at a size where finite differences
are cheap: exchange + interfacial DMI (per-cell D) + uniaxial anisotropy
(per-cell Ku) + Zeeman + demag, per-cell Ms, seeded random m0; loss
L = sum |m_T - m_target|^2 after nsteps RK4 steps."""
import numpy as np
import pytest

from helpers import GpuSim

pytestmark = pytest.mark.gpu

FD_TOL = 1e-4      # max |g_adjoint - g_fd| / max |g_fd| per parameter kind
F32_TOL = 2e-3     # FP32-form adjoint vs FP64-form adjoint, same measure
NX, NY, NZ = 24, 20, 2
DT, NSTEPS = 5e-14, 200


def _cfg(seed=104):
    rng = np.random.default_rng(seed)
    n = NX * NY * NZ
    m = rng.normal(size=(n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    t = rng.normal(size=(n, 3))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    cfg = dict(nx=NX, ny=NY, nz=NZ, dx=2e-9, dy=2e-9, dz=2e-9, pbc="", Ms=rng.uniform(6e5, 9e5, n),
               m=m.reshape(-1), terms=["exch", "dmi_int", "anis", "zeeman", "demag"], A=1.3e-11,
               Dint=rng.uniform(1e-3, 4e-3, n), Ku=rng.uniform(2e5, 5e5, n), axis=(0, 0, 1),
               H=np.tile([2e4, -1e4, 3e4], n), alpha=0.1, gamma=2.211e5)
    return cfg, t.reshape(-1)


def _tensor(cfg):
    from oracle.oracle import demag_tensor

    return demag_tensor(cfg["nx"], cfg["ny"], cfg["nz"], cfg["dx"], cfg["dy"], cfg["dz"])


def _loss(cfg, target, T, form=0):
    g = GpuSim(cfg, form=form, tensor=T)
    g.rk4(DT, NSTEPS)
    mT = g.m()
    g.h.close()
    return float(np.sum((mT - target) ** 2))


def _adjoint(cfg, target, T, form=0, ckpt=50):
    g = GpuSim(cfg, form=form, tensor=T)
    g.h.call("mm_adjoint_record", DT, NSTEPS, ckpt)
    mT = g.m()
    n = g.n
    out = {k: np.zeros(3 * n if k == "m0" else n) for k in ("m0", "Ms", "Ku", "D")}
    dp = g.lib.dptr
    g.h.call("mm_adjoint_backward", dp(np.ascontiguousarray(2 * (mT - target))), dp(out["m0"]), dp(out["Ms"]),
             dp(out["Ku"]), dp(out["D"]))
    out["mT_after"] = g.m()
    out["mT"] = mT
    g.h.close()
    return out


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cfg, target = _cfg()
    T = _tensor(cfg)
    return cfg, target, T, _adjoint(cfg, target, T)


def test_adjoint_vs_finite_differences(setup):
    cfg, target, T, adj = setup
    np.testing.assert_array_equal(adj["mT_after"], adj["mT"])  # m is left at m_T
    rng = np.random.default_rng(7)
    n = NX * NY * NZ
    checks = {"m0": ("m", rng.choice(3 * n, 8, replace=False), 1e-6),
              "Ms": ("Ms", rng.choice(n, 8, replace=False), 1e-6),
              "Ku": ("Ku", rng.choice(n, 8, replace=False), 1e-6),
              "D": ("Dint", rng.choice(n, 8, replace=False), 1e-6)}
    for kind, (key, idx, rel) in checks.items():
        fd = []
        for i in idx:
            h = rel * (1.0 if kind == "m0" else abs(cfg[key][i]))
            vals = []
            for s in (+1, -1):
                c = dict(cfg)
                c[key] = np.array(cfg[key], dtype=np.float64).copy()
                c[key][i] += s * h
                vals.append(_loss(c, target, T))
            fd.append((vals[0] - vals[1]) / (2 * h))
        fd = np.array(fd)
        ad = adj[kind][idx]
        err = np.max(np.abs(ad - fd)) / np.max(np.abs(fd))
        print(f"adjoint vs FD, {kind}: max rel err {err:.2e} (|g| up to {np.max(np.abs(fd)):.3e})")
        assert err <= FD_TOL, (kind, ad, fd)


def test_adjoint_checkpoint_interval_invariance(setup):
    """The backward sweep recomputes the same forward states whatever the
    checkpoint spacing, so the gradients are identical."""
    cfg, target, T, adj = setup
    for ck in (1, 37, NSTEPS):
        other = _adjoint(cfg, target, T, ckpt=ck)
        for k in ("m0", "Ms", "Ku", "D"):
            np.testing.assert_array_equal(other[k], adj[k])


def test_adjoint_fp32_form(setup):
    cfg, target, T, adj = setup
    a32 = _adjoint(cfg, target, T, form=1)
    for k in ("m0", "Ms", "Ku", "D"):
        err = np.max(np.abs(a32[k] - adj[k])) / np.max(np.abs(adj[k]))
        print(f"FP32 vs FP64 adjoint, {k}: {err:.2e}")
        assert err <= F32_TOL
