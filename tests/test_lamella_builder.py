"""The lamella initial state (CLamellaBuilder::Assemble, LamellaBuilder.cpp:
126-1010, with the 2-d Maxwell velocities of CBuilder::AssignMaxwellVelocities,
Builder.cpp:4207-4330) on the CPU: the oracle's restatement
(dpdo_lamella_state) against the state the unmodified reference builds
(tests/golden/lamella_*.npz, made by tests/golden/make_lamella_golden.py), bit
for bit, for normals x, y and z, straight and scattered chains and a single
monolayer; and the properties the builder guarantees (beads inside the box,
zero momentum, in-plane temperature kT, no velocity along the normal)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import dpd_oracle as O  # noqa: E402

CASES = ["lamella_z_straight", "lamella_x_straight", "lamella_y_scattered", "lamella_z_upper_only"]


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


def build(g):
    return O.lamella_state(g["L"], float(g["kT"]), int(g["seed"]), g["poly_first"], g["poly_type"],
                           int(g["lipid_type"]), int(g["head_offset"]), int(g["tail_offset"]), int(g["normal"]),
                           float(g["centre"]), float(g["thickness"]), bool(g["linearise"]),
                           float(g["upper_fraction"]), 0, g["bond_head"], g["bond_tail"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_bit_for_bit(name):
    g = load(name)
    x, v = build(g)
    assert np.array_equal(x, g["x"])
    assert np.array_equal(g["unpbc"], g["x"])   # the builder sets unPBC = x
    assert np.array_equal(v, g["v"])


@pytest.mark.parametrize("name", CASES)
def test_builder_properties(name):
    g = load(name)
    n = len(g["ids"])
    nrm = int(g["normal"])
    assert ((g["x"] >= 0.0) & (g["x"] < g["L"])).all()
    assert np.abs(g["v"].sum(axis=0)).max() < 1e-9 * n
    assert (g["v"][:, nrm] == 0.0).all()
    assert abs((g["v"] ** 2).sum() / (2 * n) - float(g["kT"])) < 1e-12
    # bilayer heads on the head planes, tails next to the mid-plane
    first, ptype = g["poly_first"], g["poly_type"]
    lip = first[:-1][ptype == int(g["lipid_type"])]
    c = float(g["centre"]) * g["L"][nrm]
    heads = g["x"][lip + int(g["head_offset"]), nrm]
    tails = g["x"][lip + int(g["tail_offset"]), nrm]
    assert np.all(np.isclose(np.abs(heads - c), 0.5 * float(g["thickness"])) | np.isclose(heads, c))
    assert np.allclose(np.abs(tails - c), 0.2)


def test_lattice_outside_the_box_is_an_error():
    g = load("lamella_z_straight")
    with pytest.raises(ValueError):
        O.lamella_state(g["L"], 1.0, 1, g["poly_first"], g["poly_type"], 0, 0, 8, 2, 0.5, 12.0, True, 0.5)


def test_control_file_lamella_block(tmp_path):
    """workloads.lamella_block: the State lamella block of a control data
    file as CInitialStateLamella reads it (InitialStateLamella.cpp), in place
    of State random."""
    sys.path.insert(0, os.path.dirname(HERE))
    from osprey_dpd_b200 import workloads as W
    s = W.bilayer(cells=(8, 8, 12), nlipids=40)
    path = tmp_path / "dmpci.t"
    W.write_dmpci(s, str(path), 10, state=W.lamella_block("Lipid", normal=(0, 1, 0), centre=0.4, thickness=4.5,
                                                         linearise=False, upper_fraction=0.25))
    text = path.read_text().split("\n")
    k = text.index("State\tlamella")
    body = [t.split() for t in text[k + 1:k + 8]]
    assert body == [["Polymer", "Lipid"], ["Normal", "0", "1", "0"], ["Centre", "0.4"], ["Thickness", "4.5"],
                    ["Linearise", "0"], ["UpperFraction", "0.25"], ["Polymerise", "0"]]
    assert "State\trandom" not in text
