"""The oracle's accurate Newell tensor against 60-digit values
(tests/golden/newell_hp.json, made by tests/golden/make_newell_hp.py).

The 27-point second differences of demag_tensor_xx / _xy
(MicroMagnetic.jl src/micro/demag.jl:194-296) cancel up to R^6 of the
function values (5e10 at R = 60 cells).  The oracle evaluates f and g in
binary128 at exact coordinates, so its entries must round correctly to FP64;
the FP64 arithmetic of the reference itself is off by up to ~1e-6 relative in
the entries near the dipole switch, which the last test measures.
"""
import json
import os
from decimal import Decimal, getcontext

import numpy as np
import pytest

from oracle.oracle import demag_tensor, newell_fn

getcontext().prec = 60  # the fixture's precision; Decimal sums below are exact
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "newell_hp.json")
CASES = json.load(open(GOLD))["cases"]


def _dec(hi_lo):
    return Decimal(hi_lo[0]) + Decimal(hi_lo[1])


@pytest.mark.parametrize("case", CASES[::3], ids=lambda c: "%s-c%d-%d.%d.%d" % (c["cell"], c["c"], c["X"], c["Y"], c["Z"]))
def test_binary128_functions(case):
    """f / g at the grid point in binary128: relative to the size of their
    terms (R^3), within 1e-31."""
    d = case["d"]
    got = _dec(newell_fn(case["c"], case["X"], case["Y"], case["Z"], *d))
    want = Decimal(case["fn"])
    R = (case["X"] ** 2 * d[0] ** 2 + case["Y"] ** 2 * d[1] ** 2 + case["Z"] ** 2 * d[2] ** 2) ** 0.5
    scale = Decimal(max(R, 1.0) ** 3)
    assert abs(got - want) <= Decimal("1e-31") * scale, (got, want)


def _mesh_entry(case, accurate):
    X, Y, Z = case["X"], case["Y"], case["Z"]
    d = case["d"]
    T = demag_tensor(X + 1, Y + 1, Z + 1, d[0], d[1], d[2], accurate=accurate)
    return T[case["c"], -1]  # the last cell of the mesh is offset (X, Y, Z)


def test_tensor_entries_round_correctly():
    """Every entry of the accurate tensor is the 60-digit value rounded to
    FP64, to within one unit in the last place (entries that vanish by
    symmetry, e.g. xy at X = 0, to within 1e-30 absolute)."""
    worst = 0.0
    for case in CASES:
        want = float(Decimal(case["entry"]))
        got = _mesh_entry(case, True)
        ulp = np.spacing(abs(want)) if abs(want) > 1e-30 else 1e-30
        assert abs(got - want) <= ulp, (case, got, want)
        if abs(want) > 1e-30:
            worst = max(worst, abs(got - want) / abs(want))
    assert worst <= 2.3e-16


def test_reference_arithmetic_error_near_dipole_switch():
    """The FP64 arithmetic of the reference loses the digits the differences
    cancel: measured against the 60-digit entries it is far from correctly
    rounded near R = 60 cells, while the accurate tensor is."""
    rel = []
    for case in CASES:
        if case["X"] < 40:
            continue
        want = float(Decimal(case["entry"]))
        if abs(want) < 1e-30:
            continue
        got = _mesh_entry(case, False)
        rel.append(abs(got - want) / abs(want))
    assert rel and 1e-12 < max(rel) < 1e-3, max(rel)
