"""The Paraview snapshot format (dpd_write_paraview, host code of the engine
library, no GPU needed) against the reference's own files
(tests/golden/paraview_*.npz, made by tests/golden/make_paraview_golden.py):
given the reference's beads in the reference's file order, the library
writes the reference's file byte for byte; and the reference's order is
cell-major (CSimBox::GetAllBeadsInCNTCells), the order the engine's writer
reproduces cell by cell."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["paraview_water_4", "paraview_polymer_6"]


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


@pytest.mark.parametrize("name", CASES)
def test_writer_reproduces_reference_file(engine_mod, name, tmp_path):
    g = load(name)
    by_id = {int(i): k for k, i in enumerate(g["id"])}
    rows = np.array([by_id[int(i)] for i in g["file_ids"]])
    path = tmp_path / "snap.vtk"
    engine_mod.write_paraview(str(path), g["x"][rows], g["type"][rows])
    assert path.read_bytes() == g["vtk"].tobytes()


@pytest.mark.parametrize("name", CASES)
def test_reference_order_is_cell_major(name):
    g = load(name)
    by_id = {int(i): k for k, i in enumerate(g["id"])}
    x = g["x"][[by_id[int(i)] for i in g["file_ids"]]]
    c, w = g["cells"], g["widths"]
    ix = (x / w).astype(np.int64)
    cell = ix[:, 0] + c[0] * (ix[:, 1] + c[1] * ix[:, 2])
    assert (np.diff(cell) >= 0).all()
