"""Bulk copies of the FP32 register path wait on an mbarrier a bounded number
of tries: the y passes for ny = 1024 (a padded y line of 2048 values arrives
in shared memory by cp.async.bulk) and the z convolution for Pz = 32 with
column-major spectra (the block's tensor slice arrives by one tiled copy
through a tensor map).  A wait that runs out makes the pass leave early
instead of hanging the GPU, and the handle reports it: mm_synchronize
returns MM_ERR_TIMEOUT (-5) and names the pass.

MMCUDA_COPY_SPINS=0 gives every first wait zero tries, so every block takes
the timeout path (it still waits, with a fixed bound, for its copy in
flight before it leaves).  The limit is read once per process, so the check
runs in a child process."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATHS = [ROOT, os.path.join(ROOT, "micromagnetic.jl_b200"), os.path.dirname(os.path.abspath(__file__))]


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


CHILD = """
import sys
sys.path[:0] = %r
from helpers import GpuSim, random_config
from mmcuda import _lib
cfg = random_config(7, %d, %d, %d, terms=("exch", "demag"), holes=False, spatial=False)
g = GpuSim(cfg, form=1)
L = _lib.load()
rc = L.mm_rk4_run(g.h.h, 2e-14, 2)
print("run", rc)
rc = L.mm_synchronize(g.h.h)
print("sync", rc, _lib.last_error())
rc = L.mm_synchronize(g.h.h)
print("again", rc)
"""


# (mesh, the pass named): the register path needs power-of-two padded
# lengths (nz = 16: Pz = 32).  ny = 1024 takes the bulk-copy y passes (its
# z convolution times out as well; the y pass is named first); ny = 512 the
# warp-direct y passes, so only the z convolution's wait runs out
MESHES = [((128, 1024, 16), "y"), ((128, 512, 16), "z")]


def _run(mesh, env):
    return subprocess.run([sys.executable, "-c", CHILD % ((PATHS,) + mesh)], env=dict(os.environ, **env),
                          capture_output=True, text=True, timeout=600)


@pytest.mark.parametrize("mesh,which", MESHES)
def test_copy_wait_limit_reports_timeout(mesh, which):
    r = _run(mesh, {"MMCUDA_COPY_SPINS": "0"})
    assert r.returncode == 0, r.stdout + r.stderr
    assert "run 0" in r.stdout and "sync -5" in r.stdout, r.stdout
    assert "demag %s pass: a bounded bulk-copy wait ran out" % which in r.stdout, r.stdout
    assert "again 0" in r.stdout, r.stdout  # the flag is cleared once reported


@pytest.mark.parametrize("mesh,which", MESHES)
def test_copy_wait_default_limit_is_clean(mesh, which):
    r = _run(mesh, {})
    assert r.returncode == 0, r.stdout + r.stderr
    assert "run 0" in r.stdout and "sync 0" in r.stdout, r.stdout
