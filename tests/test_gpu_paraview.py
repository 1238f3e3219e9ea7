"""dpd_engine_write_paraview against the reference's own Paraview snapshots
(tests/golden/paraview_*.npz): an engine holding the reference's state of
that step writes the same file cell by cell -- the same header, vertex list
and data lines, and in every CNT cell the same points with the same display
ids (inside a cell the reference's order is its cell-list history, the
engine's the upload order).  Type visibility and display ids as
CCurrentState applies them."""
import os

import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SYSTEMS = {"paraview_water_4": lambda: W.water(n=4), "paraview_polymer_6": lambda: W.polymer_solution(cells=(6, 6, 6))}


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


def engine_with_reference_state(engine_mod, name, precision):
    g = load(name)
    s = SYSTEMS[name]()
    eng = engine_mod.DpdEngine.from_system(s, precision=precision, topology=False)
    eng.upload_beads(g["id"], g["type"], None, g["x"], g["unpbc"], g["v"], g["f"])
    return g, eng


def sections(text: bytes, n: int):
    lines = text.decode().split("\n")
    head, pts = lines[:5], lines[5:5 + n]
    mid = lines[5 + n:5 + n + 1 + n + 3]
    ptype = lines[5 + n + 1 + n + 3:5 + n + 1 + n + 3 + n]
    rest = lines[5 + n + 1 + n + 3 + n:]
    return head, pts, mid, ptype, rest


def cell_blocks(g):
    """(start, end) of each cell's run of lines in the reference's file."""
    by_id = {int(i): k for k, i in enumerate(g["id"])}
    x = g["x"][[by_id[int(i)] for i in g["file_ids"]]]
    c, w = g["cells"], g["widths"]
    ix = (x / w).astype(np.int64)
    cell = ix[:, 0] + c[0] * (ix[:, 1] + c[1] * ix[:, 2])
    cuts = np.nonzero(np.diff(cell))[0] + 1
    edges = np.concatenate([[0], cuts, [len(cell)]])
    return list(zip(edges[:-1], edges[1:]))


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_engine_snapshot_matches_reference_by_cell(engine_mod, name, precision, tmp_path):
    g, eng = engine_with_reference_state(engine_mod, name, precision)
    path = tmp_path / "snap.vtk"
    eng.write_paraview(str(path))
    n = len(g["id"])
    gh, gp, gm, gt, gr = sections(path.read_bytes(), n)
    rh, rp, rm, rt, rr = sections(g["vtk"].tobytes(), n)
    assert gh == rh and gm == rm and gr == rr
    for a, b in cell_blocks(g):
        assert sorted(zip(gp[a:b], gt[a:b])) == sorted(zip(rp[a:b], rt[a:b]))
    eng.close()


def test_engine_snapshot_visibility_and_display_ids(engine_mod, tmp_path):
    g, eng = engine_with_reference_state(engine_mod, "paraview_polymer_6", 1)
    types = g["type"]
    vis = np.ones(int(types.max()) + 1, np.uint8)
    vis[0] = 0
    disp = (np.asarray(g["id"]) % 7).astype(np.int32)
    path = tmp_path / "snap.vtk"
    eng.write_paraview(str(path), type_visible=vis, display_id=disp)
    m = int((types != 0).sum())
    text = path.read_bytes()
    h, pts, mid, ptype, rest = sections(text, m)
    assert h[4].startswith(f"POINTS {m} double")
    shown = {"%.6g %.6g %.6g" % tuple(g["x"][k]): str(disp[k]) for k in range(len(types)) if types[k] != 0}
    assert sorted(zip(pts, ptype)) == sorted(shown.items())
    eng.close()
