"""The demag tile autotuner (DemagPlan::autotune): the tile widths it picks
change only the grouping of lines into blocks, so fields are bit-identical
to the static rule's; it reports a tile for every strided pass it tuned."""
import ctypes
import os

import numpy as np
import pytest

from helpers import GpuSim, random_config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _field(cfg, form, tune):
    old = os.environ.get("MMCUDA_AUTOTUNE")
    os.environ["MMCUDA_AUTOTUNE"] = "1" if tune else "0"
    try:
        g = GpuSim(cfg, form=form)
    finally:
        if old is None:
            del os.environ["MMCUDA_AUTOTUNE"]
        else:
            os.environ["MMCUDA_AUTOTUNE"] = old
    tiles = (ctypes.c_int * 5)()
    ms = (ctypes.c_float * 5)()
    g.h.call("mm_demag_tiles", tiles, ms)
    f = g.field()
    g.h.close()
    return f, list(tiles)


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("mesh", [(64, 48, 16, ""), (100, 80, 1, ""), (30, 20, 7, "xy"), (6, 210, 16, "")])
def test_autotuned_tiles_give_identical_fields(mesh, form):
    cfg = random_config(31, *mesh, terms=("exch", "demag"))
    f_static, t_static = _field(cfg, form, False)
    f_tuned, t_tuned = _field(cfg, form, True)
    assert t_static == [0, 0, 0, 0, 0]
    used = [2] if mesh[2] == 1 else [1, 2, 3]
    # nz = 16 pads z to 32: the register z convolution takes no tile (FP32
    # always; FP64 where the spectra are column-major, padded y = 420 here)
    if mesh[2] == 16 and (form == 1 or mesh[1] == 210):
        used.remove(2)
        assert t_tuned[2] == 0, t_tuned
    assert all(t_tuned[i] >= 1 for i in used), t_tuned
    np.testing.assert_array_equal(f_tuned, f_static)
