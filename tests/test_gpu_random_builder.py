"""dpd_engine_build_random: the random initial state of CRandomBuilder::
Assemble (RandomBuilder.cpp:71-361) built by the engine's kernels, against
the state the unmodified reference builds (tests/golden/random_*.npz) and, on
a 786k-bead box, against the oracle's restatement (itself equal to the
reference bit for bit): positions exact, velocities to 1e-12 (the device's
acos/sin/cos and tree sums against the C library and sequential sums); the
engine then holds that state and steps from it."""
import os
import sys

import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import dpd_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

SYSTEMS = {"random_water_10": lambda: W.water(n=10), "random_polymer_8": lambda: W.polymer_solution(cells=(8, 8, 8))}
VTOL = dict(rtol=1e-12, atol=1e-13)


def check_engine_state(eng, x, v):
    d = eng.download()
    assert np.array_equal(d["x"], x)
    assert np.array_equal(d["unpbc"], x)
    assert np.array_equal(d["v"], v)
    assert not d["f"].any()


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_build_random_equals_reference(engine_mod, name, precision):
    g = dict(np.load(os.path.join(HERE, "golden", name + ".npz")))
    s = SYSTEMS[name]()
    assert s.n == len(g["ids"]) and np.array_equal(s.box, g["L"])
    eng = engine_mod.DpdEngine.from_system(s, precision=precision)
    for _ in range(2):   # a second build replaces the first with the same state
        x, v = eng.build_random(g["ids"], g["types"], int(g["seed"]), 0, g["bond_head"], g["bond_tail"])
        assert np.array_equal(x, g["x"])
        np.testing.assert_allclose(v, g["v"], **VTOL)
        check_engine_state(eng, x, v)
    eng.close()


def test_build_random_large_box_and_steps(engine_mod):
    s = W.water(n=64)   # 786,432 beads
    seed = 4242
    xo, vo = O.random_state(s.n, s.box, s.kT, seed, 0)
    eng = engine_mod.DpdEngine.from_system(s, precision=0)
    x, v = eng.build_random(s.ids, s.types, seed)
    assert np.array_equal(x, xo)
    np.testing.assert_allclose(v, vo, **VTOL)
    check_engine_state(eng, x, v)
    eng.step(1, 10)
    assert eng.status() == 0
    o = eng.download()
    assert np.isfinite(o["x"]).all() and ((o["x"] >= 0) & (o["x"] < s.box)).all()
    eng.close()


def test_build_random_skip_and_errors(engine_mod):
    s = W.water(n=8)
    eng = engine_mod.DpdEngine.from_system(s, precision=0)
    x0, _ = eng.build_random(s.ids, s.types, 77)
    x1, _ = eng.build_random(s.ids[1:], s.types[1:], 77, skip=6)
    assert np.array_equal(x0[1:], x1)   # six draws per bead
    with pytest.raises(engine_mod.EngineError):
        eng.build_random(s.ids, s.types, 77, 0, [0], [s.n])   # bond bead index out of range
    with pytest.raises(engine_mod.EngineError):
        eng.build_random(s.ids, s.types, 77, 0, [3], [3])     # a bead bonded to itself
    eng.close()
