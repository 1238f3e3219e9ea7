"""The oracle's slice stress profile (CMonitor::AddBeadStress, AddBondStress,
AddBondPairStress, Monitor.cpp:1900-2755) against the live reference binary:
bit-identical per slice, per type pair / bond type / bond-pair type, after
several steps with the reference's own LCG noise.  Also pins the bond and
bond-pair type indices the workloads assign against the reference's.
Skipped where the reference harness was not built."""
import os

import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                                    "osprey_ref_driver")), reason="reference harness not built")

SYSTEMS = {
    "water": (lambda: W.water(6), 6),
    "binary": (lambda: W.binary_mixture(cells=(5, 6, 7), seed=9, a_ab=38.0, frac_a=0.3), 14),
    "bilayer_htt_phi30": (lambda: W.bilayer(cells=(8, 8, 8), nlipids=16, with_htt=True, phi0_deg=30.0, seed=11), 16),
    "polymer": (lambda: W.polymer_solution(cells=(6, 7, 8), seed=13), 5),
}


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_oracle_slice_stress_matches_live_reference(oracle_mod, name):
    make, slices = SYSTEMS[name]
    s = make()
    steps = 4
    _, _, _, ref = oracle_mod.run_reference(s, steps, rng_seed=s.seed, slices=slices)
    assert np.array_equal(ref["bond_type"], s.bond_type)
    assert np.array_equal(ref["angle_type"], s.angle_type)
    o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_LCG)
    o.set_slice_stress(slices)
    o.step(1, steps)
    got = o.slice_stress()
    assert o.slice_errors() == 0
    for k in ("pair", "bond", "bondpair"):
        assert got[k].shape == ref[k].shape, k
        assert np.array_equal(got[k], ref[k]), k
    # the profile is not trivially zero: its trace sums to the pair virial
    assert np.abs(got["pair"]).sum() > 0
