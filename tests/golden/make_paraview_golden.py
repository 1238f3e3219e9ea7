"""Generates paraview_*.npz here: the Paraview snapshot the unmodified
reference (oracle/_ref/osprey_ref_driver --paraview 1, i.e. CCurrentState +
CParaviewFormat) writes after a short run, with the full-precision state of
that step (the harness dump, by bead id) and the file's bead order as bead
ids (found by matching every point line to the dumped positions).

    python tests/golden/make_paraview_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from osprey_dpd_b200 import workloads as W  # noqa: E402
import dpd_oracle as O  # noqa: E402

STEPS = 3


def record(system):
    summ, d, _ = O.run_reference(system, STEPS, paraview=True)
    vtk = summ["paraview"]
    lines = vtk.decode().split("\n")
    n = system.n
    pts = lines[5:5 + n]
    key = {"%.6g %.6g %.6g" % tuple(d["x"][k]): int(d["id"][k]) for k in range(n)}
    if len(key) != n:
        raise RuntimeError("two beads print the same position")
    order = np.array([key[p] for p in pts], dtype=np.int64)
    return dict(vtk=np.frombuffer(vtk, dtype=np.uint8), file_ids=order, id=d["id"], type=d["type"].astype(np.int32),
                x=d["x"], unpbc=d["unpbc"], v=d["v"], f=d["f"], cells=np.asarray(system.cells, np.int64),
                widths=np.asarray(system.widths, np.float64))


def main():
    cases = {"paraview_water_4": W.water(n=4), "paraview_polymer_6": W.polymer_solution(cells=(6, 6, 6))}
    for name, system in cases.items():
        rec = record(system)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
        print(name, system.n, len(rec["vtk"]))


if __name__ == "__main__":
    main()
