"""The persistent RK4 step kernel (opt-in, MMCUDA_PERSIST=1: small meshes and
small batches run up to 256 steps a cooperative launch): the same states as
the default graphs of separate launches to rounding (the kernel bodies are
compiled into another kernel, where the compiler may contract other
multiply-adds: FP64 within 1e-12, FP32 within 1e-6), and a bounded grid
barrier -- a barrier whose wait limit runs out ends the kernel with
MM_ERR_TIMEOUT instead of hanging it.

The switches are read once per process, so the persistent path and the
one-spin barrier limit (MMCUDA_BARRIER_SPINS=1) run in child processes."""
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import GpuSim, random_config, rel_maxnorm

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATHS = [ROOT, os.path.join(ROOT, "micromagnetic.jl_b200"), os.path.dirname(os.path.abspath(__file__))]
MESHES = [(40, 24, 1, ""), (33, 17, 4, "xyz"), (64, 48, 3, "")]


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _child(code, env, tmp_path):
    script = tmp_path / "child.py"
    script.write_text("import sys; sys.path[:0] = %r\n" % (PATHS,) + code)
    r = subprocess.run([sys.executable, str(script)], env=dict(os.environ, **env), capture_output=True, text=True,
                       timeout=600)
    return r


STEP = """
import numpy as np
from helpers import GpuSim, random_config
out = {}
for mesh in %r:
    for form in (0, 1):
        cfg = random_config(9 + mesh[0], *mesh, terms=("exch", "dmi_int", "anis", "zeeman", "demag"))
        g = GpuSim(cfg, form=form)
        g.rk4(2e-14, 7)
        out["%%d_%%d_%%d_%%d" %% (mesh[0], mesh[1], mesh[2], form)] = g.m()
np.savez(%r, **out)
"""


def test_persistent_equals_graph(tmp_path):
    """RK4 steps of small meshes (films, 3-D, PBC; both forms) in the
    persistent kernel (a child with MMCUDA_PERSIST=1) and as separate
    launches (this process): the same states to rounding."""
    path = str(tmp_path / "persist.npz")
    r = _child(STEP % (MESHES, path), {"MMCUDA_PERSIST": "1"}, tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = np.load(path)
    for mesh in MESHES:
        for form in (0, 1):
            cfg = random_config(9 + mesh[0], *mesh, terms=("exch", "dmi_int", "anis", "zeeman", "demag"))
            g = GpuSim(cfg, form=form)
            g.rk4(2e-14, 7)
            key = "%d_%d_%d_%d" % (mesh[0], mesh[1], mesh[2], form)
            assert rel_maxnorm(g.m(), ref[key]) <= (1e-12 if form == 0 else 1e-6), (key, rel_maxnorm(g.m(), ref[key]))


BATCH = """
import numpy as np
from helpers import GpuSim, random_config, rel_maxnorm
from mmcuda import _lib
rng = np.random.default_rng(5)
pairs = []
for f in range(6):
    nx, ny, nz = int(rng.integers(8, 40)), int(rng.integers(8, 40)), int(rng.integers(1, 5))
    cfg = random_config(500 + f, nx, ny, nz, "", terms=("exch", "dmi_int", "anis", "zeeman", "demag"))
    pairs.append((GpuSim(cfg, form=1), GpuSim(cfg, form=1)))
batch = _lib.Batch([b.h for _, b in pairs])
for a, _ in pairs:
    a.rk4(2e-14, 5)
batch.rk4_run(2e-14, 5)
assert batch.launches() == (1, len(pairs)), batch.launches()
for a, b in pairs:
    assert rel_maxnorm(b.m(), a.m()) <= 1e-6, rel_maxnorm(b.m(), a.m())
print("ok")
"""


def test_persistent_batch(tmp_path):
    """A small batch (FP32) runs as one persistent launch and gives the
    states of its handles stepped one by one, to rounding."""
    r = _child(BATCH, {"MMCUDA_PERSIST": "1"}, tmp_path)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


TIMEOUT = """
from helpers import GpuSim, random_config
from mmcuda import _lib
cfg = random_config(3, 64, 48, 3, terms=("exch", "demag"))
g = GpuSim(cfg, form=0)
rc = _lib.load().mm_rk4_run(g.h.h, 2e-14, 3)
print("rc", rc, _lib.last_error())
"""


def test_barrier_wait_limit_reports_timeout(tmp_path):
    """With a barrier wait limit of one spin the blocks that arrive early give
    up: mm_rk4_run returns MM_ERR_TIMEOUT (-5) and the process ends normally."""
    r = _child(TIMEOUT, {"MMCUDA_PERSIST": "1", "MMCUDA_BARRIER_SPINS": "1"}, tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "rc -5" in r.stdout and "grid-barrier" in r.stdout, r.stdout
