"""Properties of the dynamics themselves, on the CPU oracle (no GPU).

From a seeded random unit-vector state the LLG dynamics with exchange are
chaotic: a 1e-10 perturbation of the FP64 oracle reaches O(1) within a few
hundred RK4 steps of 1e-13 s.  Any two implementations that round
differently (FP64 vs FP64 included) therefore disagree by O(1) after 1000
steps from such a state; accuracy of the FP32 form is measured on a smooth
state instead (test_gpu_parity.py::test_fp32_form_rk4_1000_steps)."""
import numpy as np

from oracle.oracle import OracleSim


def _film(m0, H):
    nx, ny = 64, 32
    s = OracleSim(nx, ny, 1, 2.5e-9, 2.5e-9, 3e-9)
    s.set_Ms(8e5)
    s.set_m(m0.reshape(-1))
    s.set_llg(0.02, 2.211e5)
    s.add_exch(Ax=1.3e-11, Ay=1.3e-11, Az=1.3e-11)
    s.add_zeeman(H)
    s.add_demag()
    return s


def test_chaos_random_state():
    rng = np.random.default_rng(101)
    n = 64 * 32
    m = rng.normal(size=(n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    H = np.tile([1.5e4, 1.0e4, 0.0], n)
    p = m + 1e-10 * rng.normal(size=m.shape)
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    a, b = _film(m, H), _film(p, H)
    a.rk4(1e-13, 400)
    b.rk4(1e-13, 400)
    assert np.max(np.abs(a.get_m() - b.get_m())) > 1e-2  # grew by > 1e8
