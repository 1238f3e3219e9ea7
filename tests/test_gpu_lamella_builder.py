"""dpd_engine_build_lamella: the lamella initial state of CLamellaBuilder::
Assemble (LamellaBuilder.cpp:126-1010) with the in-plane Maxwell velocities of
CBuilder::AssignMaxwellVelocities (Builder.cpp:4207-4330) built by the
engine's kernels, against the state the unmodified reference builds
(tests/golden/lamella_*.npz: normals x, y, z, straight and scattered chains,
a single monolayer) and, on the 393,216-bead H3T6 bilayer box and a 6.3M-bead
box, against the oracle's restatement (itself equal to the reference bit for
bit): positions exact, velocities to 1e-12 (the device's sin/cos and tree
sums against the C library and sequential sums); the engine then holds that
state and steps from it."""
import os
import sys

import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import dpd_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = ["lamella_z_straight", "lamella_x_straight", "lamella_y_scattered", "lamella_z_upper_only"]
VTOL = dict(rtol=1e-12, atol=1e-13)


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


def engine_for(engine_mod, L, kT, types, precision=0):
    nt = int(np.max(types)) + 1
    a = np.full((nt, nt), 25.0)
    return engine_mod.DpdEngine((int(L[0]), int(L[1]), int(L[2])), (1.0, 1.0, 1.0), 0.02, 0.5, kT, a,
                                np.full((nt, nt), 4.5), 7, precision)


def layout(system):
    first, ptype = [0], []
    for t, p in enumerate(system.polymers):
        for _ in range(p.count):
            first.append(first[-1] + len(p.beads))
            ptype.append(t)
    return np.array(first, np.int64), np.array(ptype, np.int32)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_build_lamella_equals_reference(engine_mod, name, precision):
    g = load(name)
    eng = engine_for(engine_mod, g["L"], float(g["kT"]), g["types"], precision)
    for _ in range(2):   # a second build replaces the first with the same state
        x, v = eng.build_lamella(g["ids"], g["types"], g["poly_first"], g["poly_type"], int(g["lipid_type"]),
                                 int(g["head_offset"]), int(g["tail_offset"]), int(g["normal"]), float(g["centre"]),
                                 float(g["thickness"]), bool(g["linearise"]), float(g["upper_fraction"]),
                                 int(g["seed"]), 0, g["bond_head"], g["bond_tail"])
        assert np.array_equal(x, g["x"])
        np.testing.assert_allclose(v, g["v"], **VTOL)
        d = eng.download()
        assert np.array_equal(d["x"], x) and np.array_equal(d["unpbc"], x) and np.array_equal(d["v"], v)
    eng.close()


@pytest.mark.parametrize("cells,nlipids,linearise", [((64, 64, 32), 6000, True), ((128, 128, 128), 20000, False)])
def test_build_lamella_large_box_and_steps(engine_mod, cells, nlipids, linearise):
    """The benchmark's bilayer box (393,216 beads) and a 6.3M-bead box against
    the oracle; the built bilayer then steps (with its bonds and bond pairs)."""
    s = W.bilayer(cells=cells, nlipids=nlipids)
    first, ptype = layout(s)
    seed = 8080
    bh, bt = s.bond_head - 1, s.bond_tail - 1
    xo, vo = O.lamella_state(s.box, s.kT, seed, first, ptype, 0, 0, 8, 2, 0.5, 5.0, linearise, 0.5, 0, bh, bt)
    eng = engine_mod.DpdEngine.from_system(s, precision=0, topology=False)
    x, v = eng.build_lamella(s.ids, s.types, first, ptype, 0, 0, 8, 2, 0.5, 5.0, linearise, 0.5, seed, 0, bh, bt)
    assert np.array_equal(x, xo)
    np.testing.assert_allclose(v, vo, **VTOL)
    eng.upload_topology(s.bond_head, s.bond_tail, s.bond_k2, s.bond_l0, s.angle_first, s.angle_second, s.angle_k3,
                        s.angle_phi0)
    eng.step(1, 5)
    assert eng.status() == 0
    o = eng.download(stress=False)
    assert np.isfinite(o["x"]).all() and ((o["x"] >= 0) & (o["x"] < s.box)).all()
    eng.close()


def test_build_lamella_errors(engine_mod):
    g = load("lamella_z_straight")
    eng = engine_for(engine_mod, g["L"], 1.0, g["types"])
    args = [g["ids"], g["types"], g["poly_first"], g["poly_type"], 0, 0, 8]
    with pytest.raises(engine_mod.EngineError):
        eng.build_lamella(*args, 2, 0.5, 12.0)            # thicker than the box
    with pytest.raises(engine_mod.EngineError):
        eng.build_lamella(*args[:6], 9)                    # tail offset past the polymer
    with pytest.raises(engine_mod.EngineError):
        eng.build_lamella(g["ids"], g["types"], g["poly_first"][:-1], g["poly_type"][:-1], 0, 0, 8)   # beads left over
    eng.close()
