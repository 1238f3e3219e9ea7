"""The CPU oracle against the live reference binary (oracle/_ref), on systems
not covered by the fixtures: other seeds and shapes, bond pairs with a
preferred angle, both bond-pair types of the reference bilayer example.
Skipped where the reference harness was not built (it needs the reference
sources to build)."""
import os

import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                                    "osprey_ref_driver")), reason="reference harness not built")

SYSTEMS = {
    "binary_5x6x7_seed9": lambda: W.binary_mixture(cells=(5, 6, 7), seed=9, a_ab=38.0, frac_a=0.3),
    "bilayer_htt_phi30": lambda: W.bilayer(cells=(8, 8, 8), nlipids=16, with_htt=True, phi0_deg=30.0, seed=11),
    "polymer_wide_cells": lambda: W.polymer_solution(cells=(6, 7, 8), seed=13),
}


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_oracle_matches_live_reference(oracle_mod, name):
    s = SYSTEMS[name]()
    steps = 30
    _, d, topo = oracle_mod.run_reference(s, steps, topology=True, rng_seed=s.seed)
    for k in ("bond_head", "bond_tail", "angle_first", "angle_second", "angle_phi0"):
        assert np.array_equal(getattr(s, k), topo[k]) if k != "angle_phi0" else np.allclose(s.angle_phi0, topo[k])
    o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_LCG)
    o.step(1, steps)
    st = o.state()
    for k in ("x", "unpbc", "v", "f", "stress"):
        assert np.array_equal(st[k], d[k]), k


def test_reference_step_loop_timing_is_reported(oracle_mod):
    s = W.water(6)
    summary, _, _ = oracle_mod.run_reference(s, 5, dump=False)
    assert summary["beads"] == s.n and summary["steps"] == 5 and summary["run_seconds"] > 0
