"""Partition of independent meshes (ensembles, NEB images) across ranks.

Inside one effective-field evaluation the meshes of an ensemble or the images
of a NEB band exchange nothing, so they shard across GPUs with no data-path
collective: each rank advances its own subset.  The cost of one RK4 step of
a mesh is dominated by its demag FFTs, about N log2(Px Py Pz) for N cells
(the zero-padded lengths), so meshes are assigned greedily, largest first,
to the least-loaded rank (longest-processing-time rule: the heaviest rank
carries at most 4/3 of the optimum).
"""
from __future__ import annotations

import math


def padded_len(n: int, even: bool = False) -> int:
    """Smallest 7-smooth length >= 2n - 1 (even along x), as the demag plan pads."""
    if n <= 1:
        return 1
    p = 2 * n - 1
    while True:
        if not (even and p % 2):
            q = p
            for f in (2, 3, 5, 7):
                while q % f == 0:
                    q //= f
            if q == 1:
                return p
        p += 1


def step_cost(nx: int, ny: int, nz: int, demag: bool = True) -> float:
    """Relative cost of one RK4 step of an nx x ny x nz mesh."""
    n = nx * ny * nz
    if not demag:
        return float(n)
    P = padded_len(nx, True) * padded_len(ny) * padded_len(nz)
    return n * max(1.0, math.log2(P))


def partition(costs, nranks: int):
    """Indices of the meshes each rank takes: lists (one per rank), each in
    increasing index order; every index appears exactly once."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * nranks
    parts = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]
