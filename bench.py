#!/usr/bin/env python
"""Throughput benchmark of the finite-difference LLG hot path (H_eff + demag +
RK4) on B200 through libmmcuda's C ABI.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c5|c2|c1|...]
                    [--impl native|reference]

One JSON line on rank 0.  Metric: LLG cell-steps/s = cells x RK4 steps / s,
whole job (N replicas of the mesh under torchrun: the path has no exchange
step between meshes, so ranks run independent replicas, scaling "weak"), for
the FP32 form (`value`) and the FP64 form (`fp64`), with the FP32 form's
relative max-norm error of m against the FP64 form after the same steps.
`e2e`: the same metric through the C ABI with pinned host arrays, copying m
in and out every step; the FP32 form's host arrays are Float32 (sim.spin in
the reference's Float32 mode), `e2e_f64_host` repeats it with Float64 arrays.
`--impl reference` times the CPU oracle (FP64 restatement of the reference
path, all host threads) on the whole mesh of the workload for one RK4 step.

Workloads (seeded synthetic inputs, numpy PCG64):
  c5  1024x1024x16 cells, 3 nm: exchange A=1.3e-11, Ms=8e5, demag (padded
      2048x2048x32); random unit m (seed 105); alpha=0.1, gamma=2.211e5; RK4
      with dt = 5e-14 s.  The default: the configuration the metric is quoted
      on.  Its line also carries c2 with RK4 and with Dormand-Prince
      (`extra_workloads`).
  c2  256x256x64 cells, 2 nm: exchange A=1e-11, bulk DMI 3e-3, Ku=5e5 along z,
      Ms=5.8e5, demag; random unit m (seed 102); alpha=0.1, gamma=2.211e5;
      RK4 with dt = 5e-14 s (--integrator dopri: Dormand-Prince, tol 1e-6).
  c1  200x50x1, 2.5x2.5x3 nm: A=1.3e-11, Ms=8e5, demag, in-plane Zeeman
      |B| <= 30 mT (seed 101); alpha=0.02, gamma=2.211e5, dt=1e-13.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "micromagnetic.jl_b200"))
sys.path.insert(0, ROOT)

MU0 = 4 * math.pi * 1e-7

WORKLOADS = {
    "c2": dict(nx=256, ny=256, nz=64, dx=2e-9, dy=2e-9, dz=2e-9, Ms=5.8e5, A=1e-11, Dbulk=3e-3, Ku=5e5,
               axis=(0, 0, 1), demag=True, alpha=0.1, gamma=2.211e5, dt=5e-14, seed=102, zeeman=None),
    "c5": dict(nx=1024, ny=1024, nz=16, dx=3e-9, dy=3e-9, dz=3e-9, Ms=8e5, A=1.3e-11, Dbulk=None, Ku=None,
               axis=(0, 0, 1), demag=True, alpha=0.1, gamma=2.211e5, dt=5e-14, seed=105, zeeman=None),
    # profiling case of c5's layout (padded 512x2048x32: column-major spectra)
    # small enough for full ncu captures
    "c5_small": dict(nx=256, ny=1024, nz=16, dx=3e-9, dy=3e-9, dz=3e-9, Ms=8e5, A=1.3e-11, Dbulk=None, Ku=None,
                     axis=(0, 0, 1), demag=True, alpha=0.1, gamma=2.211e5, dt=5e-14, seed=105, zeeman=None),
    # profiling case of the FP64 register passes (nx = 512, ny = 1024: the
    # same x / y line lengths as c5 for y, Q = 16 for x), about 2 GB in FP64
    "c5_half": dict(nx=512, ny=1024, nz=16, dx=3e-9, dy=3e-9, dz=3e-9, Ms=8e5, A=1.3e-11, Dbulk=None, Ku=None,
                    axis=(0, 0, 1), demag=True, alpha=0.1, gamma=2.211e5, dt=5e-14, seed=105, zeeman=None),
    # profiling case of the global-memory x stages: x/2 = 16000 is beyond one
    # block's shared memory
    "long_lines": dict(nx=16000, ny=64, nz=1, dx=4e-9, dy=4e-9, dz=4e-9, Ms=8e5, A=1.3e-11, Dbulk=None, Ku=None,
                       axis=(0, 0, 1), demag=True, alpha=0.1, gamma=2.211e5, dt=5e-14, seed=110, zeeman=None),
    "c1": dict(nx=200, ny=50, nz=1, dx=2.5e-9, dy=2.5e-9, dz=3e-9, Ms=8e5, A=1.3e-11, Dbulk=None, Ku=None,
               axis=(0, 0, 1), demag=True, alpha=0.02, gamma=2.211e5, dt=1e-13, seed=101, zeeman="inplane30mT"),
    # the reference's paper benchmark (figures/cpb/fig9/bench.jl:8-31): Heun,
    # 4 nm cells, A=1e-13, demag, H=(0, 100 mT, 0), alpha 0.01, N x N x 1
    "fig9": dict(nx=1000, ny=1000, nz=1, dx=4e-9, dy=4e-9, dz=4e-9, Ms=8e5, A=1e-13, Dbulk=None, Ku=None,
                 axis=(0, 0, 1), demag=True, alpha=0.01, gamma=2.211e5, dt=1e-14, seed=109, zeeman="y100mT",
                 integrator="heun", published=9.80e8),
    "fig9_4000": dict(nx=4000, ny=4000, nz=1, dx=4e-9, dy=4e-9, dz=4e-9, Ms=8e5, A=1e-13, Dbulk=None, Ku=None,
                      axis=(0, 0, 1), demag=True, alpha=0.01, gamma=2.211e5, dt=1e-14, seed=109, zeeman="y100mT",
                      integrator="heun", published=1.045e9),
    "fig9_8000": dict(nx=8000, ny=8000, nz=1, dx=4e-9, dy=4e-9, dz=4e-9, Ms=8e5, A=1e-13, Dbulk=None, Ku=None,
                      axis=(0, 0, 1), demag=True, alpha=0.01, gamma=2.211e5, dt=1e-14, seed=109, zeeman="y100mT",
                      integrator="heun", published=1.069e9),
    "fig9_10000": dict(nx=10000, ny=10000, nz=1, dx=4e-9, dy=4e-9, dz=4e-9, Ms=8e5, A=1e-13, Dbulk=None, Ku=None,
                       axis=(0, 0, 1), demag=True, alpha=0.01, gamma=2.211e5, dt=1e-14, seed=109, zeeman="y100mT",
                       integrator="heun", published=1.008e9),
}
# batched workloads: many meshes advanced by one graph launch per RK4 step
BATCHES = {
    # 48 films, nx, ny ~ U{32..256}, nz ~ U{1..4}, 2 nm cells, interfacial DMI
    # D ~ U[1,4]e-3, Ms ~ U[4,9]e5, A ~ U[0.8,1.5]e-11, demag, random m (seed 103)
    "c3": dict(kind="films", count=48, seed=103),
    # 32 NEB images of one 128x128x1 film, m interpolated between two random states
    "c3neb": dict(kind="neb", count=32, seed=103, nx=128, ny=128),
}
# reverse-mode gradients through RK4: 128x128x4 cells at 2 nm, exchange +
# interfacial DMI + anisotropy + demag, per-cell Ms ~ U[6,9]e5, random m0
# (seed 104), 2000 RK4 steps of 5e-14 s with checkpoints every 100 steps
ADJOINT = {"c4": dict(nx=128, ny=128, nz=4, dx=2e-9, A=1.3e-11, D=3e-3, Ku=4e5, alpha=0.1, gamma=2.211e5,
                      dt=5e-14, nsteps=2000, ckpt=100, seed=104)}
# the CPU baseline times a bounded block of the same physics
CPU_SAMPLE = {"c2": (128, 128, 32), "c5": (256, 256, 16), "c5_small": (256, 256, 16), "c5_half": (256, 256, 16),
              "c1": (200, 50, 1), "long_lines": (2000, 64, 1), "fig9": (1000, 1000, 1),
              "fig9_4000": (1000, 1000, 1), "fig9_8000": (1000, 1000, 1), "fig9_10000": (1000, 1000, 1)}


def synth_inputs(w, shape=None):
    nx, ny, nz = shape or (w["nx"], w["ny"], w["nz"])
    n = nx * ny * nz
    rng = np.random.default_rng(w["seed"])
    m = rng.standard_normal((n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    H = None
    if w["zeeman"] == "inplane30mT":
        r = 0.03 * math.sqrt(rng.uniform())
        phi = rng.uniform(0, 2 * math.pi)
        H = (r * math.cos(phi) / MU0, r * math.sin(phi) / MU0, 0.0)
    elif w["zeeman"] == "y100mT":
        H = (0.0, 0.1 / MU0, 0.0)
    return m.reshape(-1), H


def setup_native(w, form, device):
    from mmcuda import _lib

    h = _lib.Handle(w["nx"], w["ny"], w["nz"], w["dx"], w["dy"], w["dz"], 0, form, device)
    m, H = synth_inputs(w)
    h.call("mm_set_Ms", None, w["Ms"])
    h.set_m(m)
    h.call("mm_set_llg", w["alpha"], w["gamma"], 1)
    h.call("mm_add_exch", None, w["A"], w["A"], w["A"])
    if w["Dbulk"]:
        h.call("mm_add_dmi_bulk", w["Dbulk"], w["Dbulk"], w["Dbulk"])
    if w["Ku"]:
        h.call("mm_add_anis", None, w["Ku"], *w["axis"])
    if H is not None:
        h.call("mm_add_zeeman", None, *H)
    if w["demag"]:
        h.call("mm_add_demag", 0, 0, 0)
    return h, m


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs
    (one streaming nvidia-smi process sampling every 50 ms)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self._p = None
        self._t = None

    def _read(self):
        for line in self._p.stdout:
            row = [x.strip() for x in line.split(",")]
            if len(row) >= 9:
                self.samples.append(row)

    def __enter__(self):
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                        "--format=csv,noheader,nounits", "-lms", "50"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.2)  # the first sample precedes the timed region's work
        except Exception:
            self._p = None
        return self

    def __exit__(self, *a):
        if self._p is not None:
            time.sleep(0.1)
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except Exception:
                self._p.kill()
            self._t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and "Active" in s[5 + i]
                          and "Not" not in s[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def batch_specs(wname):
    """The meshes of a batched workload (seeded), independent of the rank count."""
    spec = BATCHES[wname]
    rng = np.random.default_rng(spec["seed"])
    out = []
    if spec["kind"] == "films":
        for _ in range(spec["count"]):
            nx, ny, nz = int(rng.integers(32, 257)), int(rng.integers(32, 257)), int(rng.integers(1, 5))
            D, Ms, A = rng.uniform(1e-3, 4e-3), rng.uniform(4e5, 9e5), rng.uniform(0.8e-11, 1.5e-11)
            m = rng.standard_normal((nx * ny * nz, 3))
            m /= np.linalg.norm(m, axis=1, keepdims=True)
            out.append(dict(nx=nx, ny=ny, nz=nz, D=D, Ms=Ms, A=A, m=m.reshape(-1)))
    else:
        nx, ny = spec["nx"], spec["ny"]
        n = nx * ny
        m1 = rng.standard_normal((n, 3))
        m2 = rng.standard_normal((n, 3))
        for k in range(spec["count"]):
            s = k / (spec["count"] - 1)
            m = (1 - s) * m1 / np.linalg.norm(m1, axis=1, keepdims=True) + s * m2 / np.linalg.norm(m2, axis=1, keepdims=True)
            m /= np.linalg.norm(m, axis=1, keepdims=True)
            out.append(dict(nx=nx, ny=ny, nz=1, D=2e-3, Ms=8e5, A=1.3e-11, m=m.reshape(-1)))
    return out


def setup_batch(wname, form, device, rank=0, ws=1):
    """Handles of this rank's share of a batched workload (meshes partitioned
    across ranks by demag-FFT cost), its cells and the whole job's cells."""
    from mmcuda import _lib
    from mmcuda.shard import partition, step_cost

    specs = batch_specs(wname)
    mine = partition([step_cost(s["nx"], s["ny"], s["nz"]) for s in specs], ws)[rank]
    handles, cells = [], 0
    for i in mine:
        s = specs[i]
        h = _lib.Handle(s["nx"], s["ny"], s["nz"], 2e-9, 2e-9, 2e-9, 0, form, device)
        h.call("mm_set_Ms", None, s["Ms"])
        h.set_m(s["m"])
        h.call("mm_set_llg", 0.1, 2.211e5, 1)
        h.call("mm_add_exch", None, s["A"], s["A"], s["A"])
        h.call("mm_add_dmi_interfacial", None, s["D"])
        h.call("mm_add_demag", 0, 0, 0)
        handles.append(h)
        cells += s["nx"] * s["ny"] * s["nz"]
    total = sum(s["nx"] * s["ny"] * s["nz"] for s in specs)
    return handles, cells, total


def run_batch(args, rank, ws, device, dist):
    import torch
    from mmcuda import _lib

    wname = args.workload
    out = {}
    for fname, form in (("fp32", _lib.MM_FP32), ("fp64", _lib.MM_FP64)):
        if args.only and fname != args.only:
            continue
        handles, cells, total = setup_batch(wname, form, device, rank, ws)
        b = _lib.Batch(handles)
        b.rk4_run(5e-14, args.warmup)
        stream = torch.cuda.ExternalStream(b.stream(), device=device)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.rk4_run(5e-14, args.steps)
        e1.record(stream)
        e1.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], device=f"cuda:{device}")
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        launches, merged = b.launches()
        out[fname] = {"value": total * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                      "instances": len(batch_specs(wname)), "cells": total, "rank0_instances": len(handles),
                      "launches_per_step": launches, "merged_instances": merged,
                      "launches_per_step_unmerged": sum(h.rk4_launches() for h in handles)}
        b.close()
        for h in handles:
            h.close()
    if rank == 0:
        r = out.get("fp32") or out.get("fp64")
        line = {"metric": "LLG cell-steps/s (H_eff+demag+RK4), batched", "value": r["value"], "unit": "cell-steps/s",
                "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f32" if "fp32" in out else "f64", "data": "synthetic (seeded numpy PCG64)",
                "config": {"workload": f"{wname}: {r['instances']} meshes, {r['cells']} cells, one graph per step, "
                                       f"{r['launches_per_step']} launches per step",
                           "parallelism": f"meshes partitioned over {ws} rank(s) by FFT cost, no collective"},
                "forms": out}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_adjoint(args, rank, ws, device, dist):
    """Gradient of L = sum |m_T - target|^2 through the workload's RK4 steps:
    mm_adjoint_record (forward with checkpoints) + mm_adjoint_backward,
    timed with CUDA events; value = cells x steps / (record + backward)."""
    import torch
    from mmcuda import _lib

    w = ADJOINT[args.workload]
    n = w["nx"] * w["ny"] * w["nz"]
    rng = np.random.default_rng(w["seed"])
    m0 = rng.standard_normal((n, 3))
    m0 /= np.linalg.norm(m0, axis=1, keepdims=True)
    target = rng.standard_normal((n, 3))
    target /= np.linalg.norm(target, axis=1, keepdims=True)
    Ms = rng.uniform(6e5, 9e5, n)
    out = {}
    for fname, form in (("fp32", _lib.MM_FP32), ("fp64", _lib.MM_FP64)):
        if args.only and fname != args.only:
            continue
        h = _lib.Handle(w["nx"], w["ny"], w["nz"], w["dx"], w["dx"], w["dx"], 0, form, device)
        h.call("mm_set_Ms", _lib.dptr(Ms), 0.0)
        h.call("mm_set_llg", w["alpha"], w["gamma"], 1)
        h.call("mm_add_exch", None, w["A"], w["A"], w["A"])
        h.call("mm_add_dmi_interfacial", None, w["D"])
        h.call("mm_add_anis", None, w["Ku"], 0.0, 0.0, 1.0)
        h.call("mm_add_demag", 0, 0, 0)
        stream = torch.cuda.ExternalStream(h.stream(), device=device)
        gm0, gMs, gKu, gD = np.zeros(3 * n), np.zeros(n), np.zeros(n), np.zeros(n)
        d = _lib.dptr
        times = []
        for rep in range(2):  # the first pass warms up (graphs, buffers)
            h.set_m(m0.reshape(-1))
            h.call("mm_synchronize")
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            h.call("mm_adjoint_record", w["dt"], w["nsteps"], w["ckpt"])
            e1.record(stream)
            mT = h.get_m()
            gT = np.ascontiguousarray(2 * (mT - target.reshape(-1)))
            e1b = torch.cuda.Event(enable_timing=True)
            e1b.record(stream)
            h.call("mm_adjoint_backward", d(gT), d(gm0), d(gMs), d(gKu), d(gD))
            e2.record(stream)
            e2.synchronize()
            times.append((e0.elapsed_time(e1), e1b.elapsed_time(e2)))
        t_rec, t_back = times[-1]
        t = torch.tensor([t_rec + t_back], device=f"cuda:{device}")
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        out[fname] = {"value": ws * n * w["nsteps"] / (ms / 1e3), "ms_record": t_rec, "ms_backward": t_back,
                      "backward_over_forward": t_back / t_rec, "dL_dD": float(gD.sum())}
        h.close()
        del stream
    if rank == 0:
        r = out.get("fp32") or out.get("fp64")
        line = {"metric": "adjoint cell-steps/s (RK4 record + backward)", "value": r["value"],
                "unit": "cell-steps/s", "n_gpus": ws, "steps": w["nsteps"], "warmup": 1,
                "ms_per_step": (r["ms_record"] + r["ms_backward"]) / w["nsteps"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32" if "fp32" in out else "f64",
                "data": "synthetic (seeded numpy PCG64)",
                "config": {"workload": f"{args.workload}: {w['nx']}x{w['ny']}x{w['nz']} exch + interfacial DMI + anis "
                                       f"+ demag, {w['nsteps']} RK4 steps, checkpoints every {w['ckpt']}"},
                "forms": out}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def cpu_baseline(wname, steps=1, full=False):
    """FP64 oracle (CPU restatement of the reference path), all host threads.
    full=False: a bounded block of the workload's physics, one warm-up step
    and `steps` timed steps.  full=True: the whole mesh of the workload, one
    warm-up field evaluation (page-in of every buffer) and `steps` timed
    steps."""
    from oracle.oracle import OracleSim, max_threads

    w = WORKLOADS[wname]
    shape = (w["nx"], w["ny"], w["nz"]) if full else CPU_SAMPLE[wname]
    nx, ny, nz = shape
    m, H = synth_inputs(w, shape)
    n = nx * ny * nz
    t_setup = time.perf_counter()
    s = OracleSim(nx, ny, nz, w["dx"], w["dy"], w["dz"])
    s.set_Ms(w["Ms"])
    s.set_m(m)
    s.set_llg(w["alpha"], w["gamma"])
    s.add_exch(Ax=w["A"], Ay=w["A"], Az=w["A"])
    if w["Dbulk"]:
        s.add_dmi_bulk(w["Dbulk"], w["Dbulk"], w["Dbulk"])
    if w["Ku"]:
        s.add_anis(np.full(n, w["Ku"]), w["axis"])
    if H is not None:
        s.add_zeeman(np.asarray(H))
    if w["demag"]:
        s.add_demag()
    t_setup = time.perf_counter() - t_setup
    heun = w.get("integrator") == "heun"
    step = s.heun if heun else s.rk4
    if full:
        s.effective_field()  # warm-up: plans and pages
    else:
        step(w["dt"], 1)  # warm-up (plans, pages)
    t0 = time.perf_counter()
    step(w["dt"], steps)
    dt = time.perf_counter() - t0
    evals = 2 if heun else 1
    what = f"the full {nx}x{ny}x{nz} {wname} mesh" if full else f"{nx}x{ny}x{nz} block of the {wname} physics"
    warm = "1 warm-up field evaluation" if full else "1 warm-up step"
    return {"value": evals * n * steps / dt, "unit": "cell-evals/s" if heun else "cell-steps/s",
            "cores": max_threads(), "kind": "port", "ms_per_step": 1e3 * dt / steps,
            "sample": f"{what}, FP64, {steps} {'Heun' if heun else 'RK4'} step(s) after {warm}, "
                      f"{dt:.1f} s timed ({t_setup:.1f} s set-up untimed)"}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import datetime

    import torch
    import torch.distributed as dist

    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, ws, local, dist


def measured_peak():
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp64_kernels(res, peak):
    """The FP64 form's per-kernel CUDA-event times and its step's fraction of
    the measured bandwidth (absent in --quick runs)."""
    kern = res.get("kernels")
    if not kern:
        return {}
    step = kern.get("rk4_step", {})
    return {"step_roofline": {"alg_bytes": step.get("alg_bytes"), "ms": step.get("ms"), "GBps": step.get("GBps"),
                              "frac": (step.get("GBps") or 0) / peak},
            "kernels": {k: {"ms": round(v["ms"], 5), "GBps": round(v["GBps"] or 0, 1), "frac": round((v["GBps"] or 0) / peak, 3)}
                        for k, v in kern.items()}}


def profiled_traffic(wname, form_name):
    """ncu DRAM bytes per launch of each kernel, from the committed summary."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        return d.get(f"{wname}/{form_name}", {})
    except Exception:
        return {}


def run_reference(args):
    rank, ws, local, dist = dist_init()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    wname = args.workload
    if wname not in WORKLOADS:
        print(json.dumps({"impl": "reference", "unavailable": f"{wname}: the CPU port times single-mesh RK4 "
                                                               "workloads only (c1, c2, c5, fig9)"}), flush=True)
        return
    w = WORKLOADS[wname]
    # the whole mesh of the workload, one timed step (bounded: a full-size
    # FP64 step of c5 takes about a minute on 16 host cores)
    base = cpu_baseline(wname, 1, full=True)
    v = base["value"]
    n = w["nx"] * w["ny"] * w["nz"]
    heun = w.get("integrator") == "heun"
    line = {"metric": ("LLG cell-evals/s (H_eff+demag+Heun, 2 evals per step)" if heun
                       else "LLG cell-steps/s (H_eff+demag+RK4), FP32 vs FP64 form at \u22641e-5 err"),
            "value": v, "unit": base["unit"], "n_gpus": args.gpus,
            "steps": 1, "warmup": 1, "ms_per_step": base["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded numpy PCG64)",
            "config": {"workload": f"{wname}: {w['nx']}x{w['ny']}x{w['nz']} {'Heun' if heun else 'RK4'}",
                       "form": "fp64", "sample": base["sample"]},
            "impl": "reference",
            "cpu_baseline": dict(base),
            "e2e": {"value": v, "unit": base["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_native(args):
    import torch

    rank, ws, local, dist = dist_init()
    device = local
    torch.cuda.set_device(device)
    from mmcuda import _lib

    wname = args.workload
    if wname in BATCHES:
        return run_batch(args, rank, ws, device, dist)
    if wname in ADJOINT:
        return run_adjoint(args, rank, ws, device, dist)
    w = WORKLOADS[wname]
    n = w["nx"] * w["ny"] * w["nz"]
    dt = w["dt"]
    forms = {"fp32": _lib.MM_FP32, "fp64": _lib.MM_FP64}
    results = {}
    integ = args.integrator or w.get("integrator", "rk4")
    if integ == "dopri":
        return run_dopri(args, w, wname, n, forms, rank, ws, device, dist)
    heun = integ == "heun"
    step_fn = "mm_heun_run" if heun else "mm_rk4_run"
    for fname in ((args.only,) if args.only else ("fp32", "fp64")):
        h, m0 = setup_native(w, forms[fname], device)
        stream = torch.cuda.ExternalStream(h.stream(), device=device)
        for _ in range(args.warmup):
            h.call(step_fn, dt, 1)
        h.call("mm_synchronize")
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(device) if fname == "fp32" else None
        if sampler:
            sampler.__enter__()
        e0.record(stream)
        h.call(step_fn, dt, args.steps)
        e1.record(stream)
        e1.synchronize()
        if sampler:
            sampler.__exit__()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        t = torch.tensor([ms], device=f"cuda:{device}")
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
        # a Heun step is two of the four field + stage passes of an RK4 step
        lps = h.rk4_launches() // 2 if heun else h.rk4_launches()
        res = {"ms_per_step": ms_max / args.steps, "value": ws * n * args.steps / (ms_max / 1e3),
               "launches_per_step": lps, "device_bytes": h.device_bytes()}
        if w["demag"]:
            tiles = (ctypes.c_int * 5)()
            h.call("mm_demag_tiles", tiles, None)
            res["tiles"] = list(tiles)
        if sampler:
            res["clocks"] = sampler.summary()
        if not heun and "fp32" in (args.only or "fp32 fp64") and "fp64" in (args.only or "fp32 fp64"):
            res["m_after"] = h.get_m()  # both forms advanced warm-up + steps from the same m0
            if not args.quick:
                # the same comparison at a fixed 50-step horizon: from the random
                # initial state the dynamics are chaotic, so any two roundings
                # (FP64 against FP64 included) part ways over hundreds of steps
                h50, _ = setup_native(w, forms[fname], device)
                h50.call(step_fn, dt, 50)
                res["m_50"] = h50.get_m()
                h50.close()
        if args.quick:
            results[fname] = res
            h.close()
            del stream
            continue
        # per-kernel CUDA-event timing on the handle's stream (same kernels as the step)
        kern = {}
        for kid, kname in enumerate(_lib.KERNELS):
            kms, kb = h.kernel_time(kid, reps=10)
            if kb > 0:
                kern[kname] = {"ms": kms, "alg_bytes": kb, "GBps": kb / (kms * 1e6) if kms > 0 else None}
        res["kernels"] = kern
        if fname == "fp32":
            # end to end through the public API with host buffers: per step,
            # H2D of m from pinned memory, one RK4 step, D2H of m.  The FP32
            # form's host arrays are Float32 (sim.spin in the reference's
            # Float32 mode: mm_set_m_f32 / mm_get_m_f32); the Float64-array
            # boundary is reported beside it
            k2 = args.steps

            def e2e(f32):
                dt_np, ct = (np.float32, ctypes.c_float) if f32 else (np.float64, ctypes.c_double)
                pin_in = torch.from_numpy(m0.astype(dt_np)).pin_memory()
                pin_out = torch.empty(3 * n, dtype=torch.float32 if f32 else torch.float64).pin_memory()
                p_in = ctypes.cast(pin_in.data_ptr(), ctypes.POINTER(ct))
                p_out = ctypes.cast(pin_out.data_ptr(), ctypes.POINTER(ct))
                set_fn, get_fn = ("mm_set_m_f32", "mm_get_m_f32") if f32 else ("mm_set_m", "mm_get_m")
                for _ in range(2):
                    h.call(set_fn, p_in)
                    h.call(step_fn, dt, 1)
                    h.call(get_fn, p_out)
                if dist is not None:
                    dist.barrier()
                torch.cuda.synchronize()
                e0.record(stream)
                for _ in range(k2):
                    h.call(set_fn, p_in)
                    h.call(step_fn, dt, 1)
                    h.call(get_fn, p_out)
                e1.record(stream)
                e1.synchronize()
                t = torch.tensor([e0.elapsed_time(e1)], device=f"cuda:{device}")
                if dist is not None:
                    dist.all_reduce(t, op=dist.ReduceOp.MAX)
                nb = (4 if f32 else 8) * 3 * n
                return {"value": ws * n * k2 / (float(t.item()) / 1e3), "unit": "cell-steps/s",
                        "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb, "steps": k2,
                        "host_dtype": "f32" if f32 else "f64"}

            res["e2e"] = e2e(True)
            res["e2e_f64_host"] = e2e(False)
        results[fname] = res
        h.close()
        del stream
    if args.quick:
        if rank == 0:
            print(json.dumps({k: {"ms_per_step": v["ms_per_step"], "value": v["value"]} for k, v in results.items()}))
        if dist is not None:
            dist.destroy_process_group()
        return
    fp32_err = None
    fp32_err_50 = None
    if "m_50" in results.get("fp32", {}) and "m_50" in results.get("fp64", {}):
        a, b = results["fp32"].pop("m_50"), results["fp64"].pop("m_50")
        fp32_err_50 = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    if "m_after" in results.get("fp32", {}) and "m_after" in results.get("fp64", {}):
        a, b = results["fp32"].pop("m_after"), results["fp64"].pop("m_after")
        fp32_err = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    extra = extra_workloads(device) if (wname == "c5" and ws == 1 and not args.no_extra) else None
    if rank == 0:
        # --only fp64 reports the FP64 form as the line's value
        main = "fp32" if "fp32" in results else "fp64"
        r = results[main]
        peak, peak_kind = measured_peak()
        kern = {k: v for k, v in r["kernels"].items() if k != "rk4_step"}
        # dominant kernel: largest time share of one RK4 step (4 launches of each)
        dom = max(kern, key=lambda k: kern[k]["ms"])
        traffic = profiled_traffic(wname, main).get(dom)
        ach = kern[dom]["alg_bytes"] / (kern[dom]["ms"] * 1e-3) / 1e9
        step = r["kernels"].get("rk4_step", {}) if not heun else {}
        # Heun is quoted per right-hand-side evaluation, two per step
        # (figures/cpb/fig9/bench.jl:28-31)
        evals = 2 if heun else 1
        unit = "cell-evals/s" if heun else "cell-steps/s"
        if heun:
            for k in ("e2e", "e2e_f64_host"):
                if k in r:
                    r[k]["value"] *= evals
                    r[k]["unit"] = unit
        line = {
            "metric": ("LLG cell-evals/s (H_eff+demag+Heun, 2 evals per step)" if heun
                       else "LLG cell-steps/s (H_eff+demag+RK4), FP32 vs FP64 form at \u22641e-5 err"),
            "value": evals * r["value"], "unit": unit, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": (evals * r["value"] / w["published"]) if w.get("published") else None,
            "dtype": "f32" if main == "fp32" else "f64", "data": "synthetic (seeded numpy PCG64)",
            "config": {"workload": f"{wname}: {w['nx']}x{w['ny']}x{w['nz']} cells, exch"
                                   + (" + bulk DMI" if w["Dbulk"] else "") + (" + anis" if w["Ku"] else "")
                                   + (" + zeeman" if w["zeeman"] else "") + " + demag, "
                                   + ("Heun" if heun else "RK4") + " dt=%g" % dt,
                       "form": ("fp32 (compensated RK state; fp64 tensor/energies)" if main == "fp32" else "fp64"),
                       "demag_tiles_autotuned": r.get("tiles"),
                       "parallelism": f"replicas x{ws}", "l2": "working set > 126 MB L2 (inputs larger than L2)"},
            "e2e": r.get("e2e"),
            "e2e_f64_host": r.get("e2e_f64_host"),
            "gpu_launches": r["launches_per_step"] * args.steps,
            "fp64": ({"value": evals * results["fp64"]["value"], "ms_per_step": results["fp64"]["ms_per_step"],
                      "fp32_over_fp64": r["value"] / results["fp64"]["value"],
                      "fp32_rel_err_vs_fp64": fp32_err, "err_after_steps": args.warmup + args.steps,
                      "fp32_rel_err_vs_fp64_50_steps": fp32_err_50,
                      **fp64_kernels(results["fp64"], peak)}
                     if "fp64" in results and main == "fp32" else None),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_kind": peak_kind,
                         "traffic": traffic},
            "step_roofline": {"alg_bytes": step.get("alg_bytes"), "ms": step.get("ms"),
                              "GBps": step.get("GBps"), "frac": (step.get("GBps") or 0) / peak},
            "kernels": {k: {"ms": round(v["ms"], 5), "GBps": round(v["GBps"] or 0, 1)} for k, v in r["kernels"].items()},
            "clocks": r.get("clocks"),
        }
        if extra:
            line["extra_workloads"] = extra
        if ws == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(wname, 1)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def time_steps(w, form, device, steps, warmup, step_fn="mm_rk4_run"):
    """CUDA-event time of `steps` fixed steps of one handle after `warmup`."""
    import torch

    h, _ = setup_native(w, form, device)
    stream = torch.cuda.ExternalStream(h.stream(), device=device)
    h.call(step_fn, w["dt"], warmup)
    h.call("mm_synchronize")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h.call(step_fn, w["dt"], steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    h.close()
    n = w["nx"] * w["ny"] * w["nz"]
    return {"value": n * steps / (ms / 1e3), "ms_per_step": ms / steps, "steps": steps}


def extra_workloads(device):
    """c2 (256x256x64, bulk DMI + anisotropy + demag) with RK4 and with
    Dormand-Prince (tol 1e-6, its own integrator), both forms, beside the c5
    headline."""
    from mmcuda import _lib

    w = WORKLOADS["c2"]
    out = {"c2_rk4": {}, "c2_dopri": {}}
    for fname, form in (("fp32", _lib.MM_FP32), ("fp64", _lib.MM_FP64)):
        out["c2_rk4"][fname] = time_steps(w, form, device, 50, 5)
        out["c2_dopri"][fname] = dopri_forms(w, {fname: form}, 10, 3, 1, device, None)[fname]
    for k in out:
        out[k]["fp32_over_fp64"] = out[k]["fp32"]["value"] / out[k]["fp64"]["value"]
    out["c2_rk4"]["workload"] = "c2: 256x256x64 exch + bulk DMI + anis + demag, RK4 dt=5e-14"
    out["c2_dopri"]["workload"] = "c2: 256x256x64 exch + bulk DMI + anis + demag, Dormand-Prince tol 1e-6"
    return out


def dopri_forms(w, forms, steps, warmup, ws, device, dist):
    """Accepted cell-steps/s of Dormand-Prince (tol 1e-6) through mm_run_until
    for each form, the step control running on the device."""
    import torch
    from mmcuda import _lib

    n = w["nx"] * w["ny"] * w["nz"]
    out = {}
    for fname, form in forms.items():
        h, _ = setup_native(w, form, device)
        h.call("mm_dopri_set_tol", 1e-6)
        st = _lib.Stats()
        L = _lib.load()
        _lib.check(L.mm_run_until(h.h, 1e-15, ctypes.byref(st)))  # initial step + first attempts
        for _ in range(warmup):
            _lib.check(L.mm_advance_step(h.h, ctypes.byref(st)))
        t0, n0, a0, r0 = st.t, st.nsteps, st.attempts, st.rejected
        span = steps * st.step_next
        stream = torch.cuda.ExternalStream(h.stream(), device=device)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(L.mm_run_until(h.h, t0 + span, ctypes.byref(st)))
        e1.record(stream)
        e1.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], device=f"cuda:{device}")
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        acc = st.nsteps - n0
        out[fname] = {"value": ws * n * acc / (ms / 1e3), "ms_per_step": ms / max(1, acc), "accepted": acc,
                      "attempts": st.attempts - a0, "rejected": st.rejected - r0, "t_span": span}
        h.close()
    return out


def run_dopri(args, w, wname, n, forms, rank, ws, device, dist):
    """Dormand-Prince (tol 1e-6) through mm_run_until: cell-steps/s over
    accepted steps, the step control running on the device."""
    sel = {k: v for k, v in forms.items() if not args.only or k == args.only}
    out = dopri_forms(w, sel, args.steps, args.warmup, ws, device, dist)
    if rank == 0:
        r = out.get("fp32") or out.get("fp64")
        line = {"metric": "LLG cell-steps/s (H_eff+demag+Dormand-Prince)", "value": r["value"], "unit": "cell-steps/s",
                "n_gpus": ws, "steps": r["accepted"], "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if "fp32" in out else "f64", "data": "synthetic (seeded numpy PCG64)",
                "config": {"workload": f"{wname}: {w['nx']}x{w['ny']}x{w['nz']} Dormand-Prince tol 1e-6"},
                "forms": out}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c5", choices=sorted(WORKLOADS) + sorted(BATCHES) + sorted(ADJOINT))
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="c5: skip the c2 RK4 / Dormand-Prince extra keys")
    ap.add_argument("--only", choices=["fp32", "fp64"], help="time one form only (profiling runs)")
    ap.add_argument("--quick", action="store_true", help="timed steps only: no e2e, kernel timing or CPU leg")
    ap.add_argument("--integrator", default=None, choices=["rk4", "heun", "dopri"],
                    help="default: the workload's own (RK4, or Heun for fig9)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_native(args)


if __name__ == "__main__":
    main()
