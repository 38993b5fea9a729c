"""Regenerate the golden fixtures in this folder from the reference's own tests.

Run from the repository root with the MicroMagnetic.jl checkout as the
argument:

    python tests/golden/make_golden.py <reference_root>

Sources (read as text; nothing of the reference is executed):
  * test/test_fields.txt + test/test_fields.jl:9-59 -> fields_20x5x3.npz
    (Fidimag-generated per-term fields and energies on a 20x5x3 mesh)
  * test/test_demag.jl:8-57 -> demag_known.json (three known-answer meshes)
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(root):
    data = np.loadtxt(os.path.join(root, "test", "test_fields.txt"), comments="#")
    N, _ = data.shape
    n_cells = (N - 1) // 3
    np.savez_compressed(
        os.path.join(HERE, "fields_20x5x3.npz"),
        Ms=data[:n_cells, 0],
        m0=data[: N - 1, 1],
        demag=data[: N - 1, 2],
        exch=data[: N - 1, 3],
        dmi=data[: N - 1, 4],
        dmi_interfacial=data[: N - 1, 5],
        anis=data[: N - 1, 6],
        energy=data[N - 1, 2:7],  # demag, exch, dmi, dmi_interfacial, anis
    )

    src = open(os.path.join(root, "test", "test_demag.jl")).read()
    body = src[src.index("function test_demag"): src.index("function test_demag_direct")]
    arrays = []
    for m in re.finditer(r"\[([-0-9.,eE\s]+)\]", body):
        vals = [float(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()]
        if len(vals) >= 6:
            arrays.append(vals)
    assert len(arrays) == 3, len(arrays)
    cases = [
        dict(nx=2, ny=1, nz=1, dx=2e-9, dy=2e-9, dz=2e-9, Ms=8.6e5, m=[1, 0, 0], field=arrays[0]),
        dict(nx=3, ny=2, nz=1, dx=1e-9, dy=1e-9, dz=1e-9, Ms=8.6e5, m=[0.1, 0.2, 1], field=arrays[1]),
        dict(nx=12, ny=1, nz=1, dx=2.0, dy=1.0, dz=1.0, Ms=8.6e5, m=[0.5, 0.6, 0.7], field=arrays[2]),
    ]
    with open(os.path.join(HERE, "demag_known.json"), "w") as f:
        json.dump(dict(source="test/test_demag.jl:8-57", cases=cases), f, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <MicroMagnetic.jl root>")
    main(sys.argv[1])
