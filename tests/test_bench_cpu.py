"""Host-side pieces of bench.py (no GPU): the FP64 kernel summary, the
committed ncu traffic figures the bench line quotes, and the workload tables."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

KERNELS = ("demag_fwd_x", "demag_fwd_y", "demag_conv", "demag_inv_y", "demag_inv_x", "rk4_stage")


def test_fp64_kernel_summary():
    peak = 6000.0
    res = {"kernels": {"demag_conv": {"ms": 2.0, "alg_bytes": 6e9, "GBps": 3000.0},
                       "rk4_step": {"ms": 10.0, "alg_bytes": 3e10, "GBps": 3000.0}}}
    out = bench.fp64_kernels(res, peak)
    assert out["step_roofline"]["frac"] == pytest.approx(0.5)
    assert out["kernels"]["demag_conv"]["frac"] == pytest.approx(0.5)
    assert bench.fp64_kernels({}, peak) == {}  # --quick runs time no kernels


@pytest.mark.parametrize("key", ["c5/fp32", "c5/fp64", "c2/fp32", "c2/fp64", "c5_small/fp32", "c5_half/fp64"])
def test_traffic_profiles_cover_the_step_kernels(key):
    """Every per-step kernel of the profiled workloads has one launch's DRAM
    bytes in profiles/traffic.json, within a factor of two of its algorithmic
    bytes at c5 (more means re-reads, less means L2-resident spectra)."""
    with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
        t = json.load(f)
    assert key in t
    for k in KERNELS:
        assert t[key][k] > 0, (key, k)
    if key.startswith("c5/"):
        w = 4 if key.endswith("fp32") else 8
        n = 1024 * 1024 * 16
        # algorithmic bytes of the z convolution at c5: 2 nY cw + 6 Ts w
        nY, Ts = 3 * 16 * 2048 * 1025, 17 * 1025 * 1025
        alg = 2 * nY * 2 * w + 6 * Ts * w
        assert 0.5 * alg < t[key]["demag_conv"] < 2.0 * alg
        assert 0.5 * 16 * n * w < t[key]["rk4_stage"] < 2.0 * 19 * n * w


def test_every_workload_has_a_cpu_sample():
    for name, w in bench.WORKLOADS.items():
        assert name in bench.CPU_SAMPLE, name
        sx, sy, sz = bench.CPU_SAMPLE[name]
        assert sx <= w["nx"] and sy <= w["ny"] and sz <= w["nz"], name
