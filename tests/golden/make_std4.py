"""Fixtures for the standard problem 4 end-to-end test (test_gpu_std4.py).

std4_oommf.npz: <m>(t) of OOMMF for mumag standard problem 4 as shipped with
MicroMagnetic.jl (docs/src/micromagnetics/assets/std4_oommf.txt), every 10 ps.
std4_oracle.npz: the same protocol run by the CPU oracle (FP64), following
docs/tutorials/micromagnetics/std4.jl: 200x50x1 cells of 2.5x2.5x3 nm,
Ms=8e5, A=1.3e-11, demag; SD relax from (1, 0.25, 0.1) to stopping_dmdt 0.01;
then LLG (alpha 0.02, gamma 2.211e5, Dormand-Prince tol 1e-6) in the field
(-24.6, 4.3, 0) mT, <m> at t = i * 10 ps, i = 0..100.

Run from the repository root with the reference checkout as the argument:
    python tests/golden/make_std4.py <MicroMagnetic.jl root>
"""
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
OOMMF_ASSET = "docs/src/micromagnetics/assets/std4_oommf.txt"  # path inside the reference checkout
MU0 = 4 * math.pi * 1e-7
mT = 1e-3 / MU0


def oommf(ref_root):
    d = np.loadtxt(os.path.join(ref_root, OOMMF_ASSET))
    keep = np.abs(np.round(d[:, 0] / 1e-11) * 1e-11 - d[:, 0]) < 1e-16
    d = d[keep]
    np.savez(os.path.join(HERE, "std4_oommf.npz"), t=d[:, 0], m=d[:, 1:4])
    print("oommf rows", len(d))


def oracle():
    from oracle.oracle import OracleSim

    nx, ny = 200, 50
    n = nx * ny
    s = OracleSim(nx, ny, 1, 2.5e-9, 2.5e-9, 3e-9)
    s.set_Ms(8e5)
    m0 = np.tile(np.array([1, 0.25, 0.1]) / np.linalg.norm([1, 0.25, 0.1]), n)
    s.set_m(m0)
    s.add_exch(Ax=1.3e-11, Ay=1.3e-11, Az=1.3e-11)
    s.add_demag()
    t0 = time.time()
    steps, dmdt = s.relax("SD", 10000, 0.01)
    print("relax steps", steps, "dmdt", dmdt, "%.1fs" % (time.time() - t0))
    m_relaxed = s.get_m()
    s.set_m(m_relaxed)       # set_driver: a new LLG integrator from sim.spin
    s.set_method(0)
    s.set_tol(1e-6)
    s.set_llg(0.02, 2.211e5)
    s.add_zeeman(np.tile([-24.6 * mT, 4.3 * mT, 0.0], n))
    ts, ms = [0.0], [m_relaxed.reshape(-1, 3).mean(axis=0)]
    for i in range(1, 101):
        ok, st = s.run_until(i * 1e-11)
        assert ok
        ts.append(i * 1e-11)
        ms.append(s.get_m().reshape(-1, 3).mean(axis=0))
        if i % 10 == 0:
            print(i, ms[-1], st["nsteps"], "%.1fs" % (time.time() - t0), flush=True)
    np.savez(os.path.join(HERE, "std4_oracle.npz"), t=np.array(ts), m=np.array(ms), relax_steps=steps,
             relax_dmdt=dmdt, m_relaxed_avg=ms[0])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_std4.py <MicroMagnetic.jl root>")
    oommf(sys.argv[1])
    oracle()
