"""High-precision Newell tensor entries: the fixture that pins the oracle's
binary128 tensor (tests/test_newell_accuracy.py).

The Newell functions f and g (MicroMagnetic.jl src/micro/demag.jl:133-192)
and the 27-point second differences of demag_tensor_xx / demag_tensor_xy
(demag.jl:194-296) are evaluated with Python's decimal module at 60
significant digits, at the exact coordinates X * dx (dx the double-precision
normalised cell size, converted to Decimal exactly).  atan is a Taylor series
after argument halving, asinh is ln(t + sqrt(t^2 + 1)) with Decimal.ln /
Decimal.sqrt, pi comes from Machin's formula.  Nothing of the reference is
read or executed.

    python tests/golden/make_newell_hp.py      (writes tests/golden/newell_hp.json)
"""
import json
import os
from decimal import Decimal, getcontext

getcontext().prec = 60
HERE = os.path.dirname(os.path.abspath(__file__))


def _atan_small(x):
    x2 = x * x
    s, t, k = Decimal(0), x, 0
    eps = Decimal(10) ** -70
    while abs(t) / (2 * k + 1) > eps:
        s += t / (2 * k + 1) if k % 2 == 0 else -t / (2 * k + 1)
        t *= x2
        k += 1
    return s


def _pi():
    return 16 * _atan_small(Decimal(1) / 5) - 4 * _atan_small(Decimal(1) / 239)


PI = _pi()


def atan(x):
    if x == 0:
        return Decimal(0)
    if x < 0:
        return -atan(-x)
    if x > 1:
        return PI / 2 - atan(1 / x)
    for _ in range(6):  # atan(x) = 2 atan(x / (1 + sqrt(1 + x^2)))
        x = x / (1 + (1 + x * x).sqrt())
    return 64 * _atan_small(x)


def asinh(t):
    if t == 0:
        return Decimal(0)
    if t < 0:
        return -asinh(-t)
    return (t + (t * t + 1).sqrt()).ln()


def newell_f(x, y, z):
    x2, y2, z2 = x * x, y * y, z * z
    R = (x2 + y2 + z2).sqrt()
    if R == 0:
        return Decimal(0)
    f = (2 * x2 - y2 - z2) * R / 6
    if x2 > 0:
        f -= x * y * z * atan(y * z / (x * R))
    if x2 + z2 > 0:
        f += y * (z2 - x2) * asinh(y / (x2 + z2).sqrt()) / 2
    if x2 + y2 > 0:
        f += z * (y2 - x2) * asinh(z / (x2 + y2).sqrt()) / 2
    return f


def newell_g(x, y, z):
    x2, y2, z2 = x * x, y * y, z * z
    R = (x2 + y2 + z2).sqrt()
    if R == 0:
        return Decimal(0)
    g = -x * y * R / 3
    if z2 > 0:
        g -= z2 * z * atan(x * y / (z * R)) / 6
    if y2 > 0:
        g -= y2 * z * atan(x * z / (y * R)) / 2
    if x2 > 0:
        g -= x2 * z * atan(y * z / (x * R)) / 2
    if x2 + y2 > 0:
        g += x * y * z * asinh(z / (x2 + y2).sqrt())
    if y2 + z2 > 0:
        g += y * (3 * z2 - y2) * asinh(x / (y2 + z2).sqrt()) / 6
    if x2 + z2 > 0:
        g += x * (3 * z2 - x2) * asinh(y / (x2 + z2).sqrt()) / 6
    return g


def fn(c, X, Y, Z, d):
    """f or g of component c (xx yy zz xy xz yz) at integer offsets, arguments
    permuted as demag_tensor_yy / zz / xz / yz do."""
    x, y, z = Decimal(X) * d[0], Decimal(Y) * d[1], Decimal(Z) * d[2]
    return [lambda: newell_f(x, y, z), lambda: newell_f(y, x, z), lambda: newell_f(z, y, x),
            lambda: newell_g(x, y, z), lambda: newell_g(x, z, y), lambda: newell_g(y, z, x)][c]()


def entry(c, X, Y, Z, d):
    s = Decimal(0)
    for a in (-1, 0, 1):
        for b in (-1, 0, 1):
            for e in (-1, 0, 1):
                w = (2 if a == 0 else -1) * (2 if b == 0 else -1) * (2 if e == 0 else -1)
                s += w * fn(c, X + a, Y + b, Z + e, d)
    return s / (4 * PI * d[0] * d[1] * d[2])


def main():
    cells = {
        "cubic": (1.0, 1.0, 1.0),
        # 2.5 x 2.5 x 3 nm normalised by the largest side, as the reference does
        "film": (2.5e-9 / 3e-9, 2.5e-9 / 3e-9, 3e-9 / 3e-9),
        "flat": (1.0, 0.8, 0.5),
    }
    offsets = [(0, 0, 0), (1, 0, 0), (3, 2, 1), (7, 5, 3), (20, 11, 2), (42, 42, 1), (59, 10, 0), (60, 0, 0),
               (35, 40, 25), (70, 10, 0)]
    out = {"source": "demag.jl:133-296 restated in Python decimal, 60 digits", "cases": []}
    for name, d in cells.items():
        dd = tuple(Decimal(v) for v in d)
        for X, Y, Z in offsets:
            R = (X * X * d[0] ** 2 + Y * Y * d[1] ** 2 + Z * Z * d[2] ** 2) ** 0.5
            if R > 60:
                continue
            for c in range(6):
                out["cases"].append({"cell": name, "d": list(d), "c": c, "X": X, "Y": Y, "Z": Z,
                                     "fn": str(fn(c, X, Y, Z, dd)), "entry": str(entry(c, X, Y, Z, dd))})
    with open(os.path.join(HERE, "newell_hp.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(len(out["cases"]), "cases")


if __name__ == "__main__":
    main()
