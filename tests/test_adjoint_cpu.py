"""The facts the RK4 adjoint kernels rest on, checked on the CPU oracle.

1. Every field term of the path is H = M^-1 K m (+ Zeeman) with K symmetric
   and M = diag(mu0 Ms): the transpose of dH/dm is then v -> M H_lin(M^-1 v),
   i.e. the same field kernels evaluated on w = v / (mu0 Ms).  Checked on the
   oracle's fields (restating src/micro/kernels.jl and src/micro/demag.jl)
   with spatial A, D, Ku, random Ms with holes and periodic boundaries.
2. The vector-Jacobian product of the LLG right-hand side (src/llg/llg.jl)
   that k_adj_rhs evaluates, restated here in numpy, matches numerical
   Jacobians of the oracle's llg_rhs.
"""
import numpy as np
import pytest

from helpers import build_oracle, random_config

MU0 = 4e-7 * np.pi


def _jacobian(fun, n3, h=1.0):
    """Columns of a linear map by unit probes (exact up to rounding)."""
    J = np.zeros((n3, n3))
    base = fun(np.zeros(n3))
    for c in range(n3):
        e = np.zeros(n3)
        e[c] = h
        J[:, c] = (fun(e) - base) / h
    return J


@pytest.mark.parametrize("term", ["exch", "dmi_bulk", "dmi_int", "anis", "demag"])
@pytest.mark.parametrize("pbc", ["", "xy"])
def test_field_operator_is_ms_weighted_symmetric(term, pbc):
    cfg = random_config(21, 4, 3, 2, pbc, holes=True, terms=(term,))
    o, idx = build_oracle(cfg)
    n = o.n
    ms3 = np.repeat(MU0 * cfg["Ms"], 3)  # AoS: the oracle's field arrays are AoS [x1,y1,z1,...]

    def field(m):
        f, _ = o.term_field(idx[term], m)
        return f

    J = _jacobian(field, 3 * n)
    MJ = ms3[:, None] * J
    scale = np.max(np.abs(MJ))
    assert scale > 0
    assert np.max(np.abs(MJ - MJ.T)) <= 1e-10 * scale


def _llg_vjp(m, h, u, alpha, C, precession=True):
    """Numpy restatement of the per-cell VJP in k_adj_rhs."""
    v = C * u
    mm = m @ m
    mh = m @ h
    p = mm * h - mh * m
    r = -alpha * v + (np.cross(v, m) if precession else 0.0)
    ae = (np.cross(p, v) if precession else np.zeros(3)) + 2 * (r @ h) * m - (r @ m) * h - mh * r
    q = mm * r - (r @ m) * m
    return ae, q


@pytest.mark.parametrize("precession", [True, False])
def test_llg_vjp_formulas(precession):
    rng = np.random.default_rng(5)
    alpha, gamma = 0.07, 2.211e5
    C = -gamma / (1 + alpha * alpha)

    def f(m, h):
        mm, mh = m @ m, m @ h
        p = mm * h - mh * m
        return C * ((np.cross(m, p) if precession else 0.0) - alpha * p)

    for _ in range(5):
        m = rng.normal(size=3)
        h = rng.normal(size=3) * 1e5
        u = rng.normal(size=3)
        ae, q = _llg_vjp(m, h, u, alpha, C, precession)
        eps = 1e-6
        Jm = np.array([(f(m + eps * e, h) - f(m - eps * e, h)) / (2 * eps) for e in np.eye(3)]).T
        Jh = np.array([(f(m, h + eps * 1e5 * e) - f(m, h - eps * 1e5 * e)) / (2 * eps * 1e5) for e in np.eye(3)]).T
        np.testing.assert_allclose(ae, Jm.T @ u, rtol=1e-7, atol=1e-9 * np.max(np.abs(Jm.T @ u)))
        np.testing.assert_allclose(q, Jh.T @ u, rtol=1e-7, atol=1e-9 * np.max(np.abs(Jh.T @ u)))


def test_llg_rhs_matches_oracle():
    """The function whose VJP is taken is the oracle's llg_rhs (one cell, pinned off)."""
    cfg = random_config(8, 1, 1, 1, "", holes=False, terms=("zeeman",))
    cfg["H"] = np.array([3e4, -2e4, 5e4])
    o, _ = build_oracle(cfg)
    m = cfg["m"]
    alpha, gamma = cfg["alpha"], cfg["gamma"]
    C = -gamma / (1 + alpha * alpha)
    h = cfg["H"]
    p = (m @ m) * h - (m @ h) * m
    np.testing.assert_allclose(o.llg_rhs(m), C * (np.cross(m, p) - alpha * p), rtol=1e-13)
