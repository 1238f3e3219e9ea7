"""The CPU oracle against golden fixtures produced by the reference itself.

tests/golden/*.npz hold the state of the unmodified Osprey-DPD binary after 25
steps of small seeded systems (thermostat on with the reference's LCG, kT = 0,
gamma = 0; water, A/B mixture, bilayer with bonds and bond pairs, polymer
melt), written by tests/golden/make_golden.py.  The oracle must reproduce every
bead bit for bit: this pins the restatement to the reference."""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _cases():
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden
    return make_golden


FIXTURES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("stats_", "restart_", "random_", "paraview_", "glue_",
                                                         "lamella_")))
# stats_*: tests/golden/make_stats.py; restart_*: tests/golden/make_restart_golden.py;
# random_*: tests/golden/make_random_golden.py; paraview_*: tests/golden/make_paraview_golden.py;
# glue_*: tests/golden/make_glue_golden.py; lamella_*: tests/golden/make_lamella_golden.py


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_reproduces_reference_fixture(oracle_mod, name):
    mg = _cases()
    make, steps, kT, gs = mg.cases()[name]
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    s = make()
    assert mg.input_checksum(s) == str(g["checksum"]), "input generator changed; regenerate the fixtures"
    assert int(g["steps"]) == steps
    o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_LCG, kT=kT, gamma_scale=gs)
    o.step(1, steps)
    st = o.state()
    for k in ("x", "unpbc", "v", "f"):
        assert np.array_equal(st[k], g[k]), k
    assert np.array_equal(st["stress"].sum(axis=0), g["stress_sum"])
    assert np.array_equal(st["stress"][:8], g["stress_first"])
    assert o.cell_errors() == 0


@pytest.mark.parametrize("name", ["bilayer_7", "polymer_7"])
def test_generator_topology_matches_reference(name):
    mg = _cases()
    s = mg.cases()[name][0]()
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    for k in ("bond_head", "bond_tail", "angle_first", "angle_second"):
        assert np.array_equal(getattr(s, k), g[k]), k
