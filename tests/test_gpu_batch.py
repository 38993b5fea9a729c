"""Batched stepping (mm_batch_*): several uneven meshes, or NEB-like images of
one mesh, advanced by one graph launch per RK4 step must give exactly the
states of the same handles stepped one by one."""
import numpy as np
import pytest

from helpers import GpuSim, random_config, rel_maxnorm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _films(seed, form):
    rng = np.random.default_rng(seed)
    sims = []
    for f in range(5):
        nx, ny, nz = int(rng.integers(8, 40)), int(rng.integers(8, 40)), int(rng.integers(1, 5))
        cfg = random_config(seed + f, nx, ny, nz, "", terms=("exch", "dmi_int", "anis", "zeeman", "demag"))
        sims.append((GpuSim(cfg, form=form), GpuSim(cfg, form=form)))
    return sims


@pytest.mark.parametrize("form", [0, 1])
def test_batch_equals_individual_steps(form):
    from mmcuda import _lib

    pairs = _films(303, form)
    batch = _lib.Batch([b.h for _, b in pairs])
    for a, _ in pairs:
        a.rk4(2e-14, 7)
    batch.rk4_run(2e-14, 7)
    for a, b in pairs:
        assert rel_maxnorm(b.m(), a.m()) == 0.0
    # the meshes' passes share launches: far fewer than one chain per mesh
    launches, merged = batch.launches()
    per_mesh = sum(b.h.rk4_launches() for _, b in pairs)
    assert merged == len(pairs) and launches < per_mesh / 2, (launches, merged, per_mesh)
    batch.close()


def test_batch_neb_images():
    """Images of one film interpolated between two states (the NEB layout)."""
    from mmcuda import _lib

    rng = np.random.default_rng(7)
    nx, ny = 24, 20
    n = nx * ny
    m1 = rng.normal(size=(n, 3))
    m2 = rng.normal(size=(n, 3))
    m1 /= np.linalg.norm(m1, axis=1, keepdims=True)
    m2 /= np.linalg.norm(m2, axis=1, keepdims=True)
    imgs = []
    for k in range(6):
        s = k / 5
        m = (1 - s) * m1 + s * m2
        m /= np.linalg.norm(m, axis=1, keepdims=True)
        cfg = dict(nx=nx, ny=ny, nz=1, dx=2e-9, dy=2e-9, dz=2e-9, pbc="", Ms=np.full(n, 8e5), m=m.reshape(-1),
                   terms=["exch", "dmi_int", "demag"], A=1.3e-11, Dint=np.full(n, 2e-3), alpha=0.1, gamma=2.211e5)
        imgs.append((GpuSim(cfg, form=0), GpuSim(cfg, form=0)))
    batch = _lib.Batch([b.h for _, b in imgs])
    batch.rk4_run(5e-14, 5)
    batch.rk4_run(5e-14, 5)
    for a, b in imgs:
        a.rk4(5e-14, 10)
        assert rel_maxnorm(b.m(), a.m()) == 0.0
    batch.close()
