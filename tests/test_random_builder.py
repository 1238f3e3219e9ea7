"""The random initial state (CRandomBuilder::Assemble, RandomBuilder.cpp:
71-361) on the CPU: the oracle's restatement (dpdo_random_state) against the
state the unmodified reference builds (tests/golden/random_*.npz, made by
tests/golden/make_random_golden.py), bit for bit, and the properties the
builder guarantees (zero total momentum, 3N-normalised temperature, beads
inside the box)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import dpd_oracle as O  # noqa: E402

CASES = ["random_water_10", "random_polymer_8"]


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_bit_for_bit(name):
    g = load(name)
    x, v = O.random_state(len(g["ids"]), g["L"], float(g["kT"]), int(g["seed"]), 0, g["bond_head"], g["bond_tail"])
    assert np.array_equal(x, g["x"])
    assert np.array_equal(g["unpbc"], g["x"])   # the builder sets unPBC = x
    assert np.array_equal(v, g["v"])


@pytest.mark.parametrize("name", CASES)
def test_builder_properties(name):
    g = load(name)
    n = len(g["ids"])
    assert ((g["x"] >= 0.0) & (g["x"] < g["L"])).all()
    assert np.abs(g["v"].sum(axis=0)).max() < 1e-9 * n
    assert abs((g["v"] ** 2).sum() / (3 * n) - float(g["kT"])) < 1e-12
    if len(g["bond_head"]):
        d = np.abs(g["x"][g["bond_tail"]] - g["x"][g["bond_head"]])
        assert (d <= 1.0 + 1e-12).all()   # every component of every bond shortened to at most 1


def test_skip_shifts_the_stream():
    g = load("random_water_10")
    x0, _ = O.random_state(200, g["L"], 1.0, int(g["seed"]), 0)
    x6, _ = O.random_state(199, g["L"], 1.0, int(g["seed"]), 6)
    assert np.array_equal(x0[1:], x6)   # six draws per bead
