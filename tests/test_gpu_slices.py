"""The engine's slice stress profile (CMonitor::AddBeadStress, AddBondStress,
AddBondPairStress, Monitor.cpp:1900-2755) against the CPU oracle, whose own
profile is pinned bit-for-bit to the reference (test_oracle_slices.py).  Both
run the Philox pair noise with the thermostat on.  Bounds, relative to the
largest bin of each part: 1e-4 for mixed precision (FP32 pair forces), 1e-9
for FP64.  Pair bins are compared as t1*T+t2 + t2*T+t1 sums, because inside
one cell the reference's bead order (hence the split between the two type
orders) is its linked-list order."""
import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "water": (lambda: W.water(8), 8),
    "binary": (lambda: W.binary_mixture(cells=(8, 9, 10)), 10),
    "bilayer": (lambda: W.bilayer(cells=(12, 12, 12), nlipids=60, with_htt=True, phi0_deg=30.0), 24),
    "polymer": (lambda: W.polymer_solution(cells=(12, 12, 12)), 6),
    # density 10: ~21 pairs a bead, more than the engine's pair list holds
    # (16 a bead), so the profile is built by its one-kernel fallback
    "water_dense": (lambda: W.water(5, density=10.0), 5),
}


def _sym(pair, T):
    out = pair.reshape(pair.shape[0], T, T, 9).copy()
    return out + out.transpose(0, 2, 1, 3)


def _close(a, b, tol):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) <= tol * scale


def _run(engine_mod, oracle_mod, s, S, precision, steps, period):
    eng = engine_mod.DpdEngine.from_system(s, precision=precision)
    eng.set_slice_stress_for(s, S)
    eng.set_sample_period(period)
    eng.step(1, steps)
    got = eng.slice_stress()
    assert eng.status() == 0
    return got


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_slice_stress_matches_oracle(engine_mod, oracle_mod, name, precision):
    make, S = SYSTEMS[name]
    s = make()
    got = _run(engine_mod, oracle_mod, s, S, precision, steps=3, period=1)
    o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    o.set_slice_stress(S)
    o.step(1, 3)
    ref = o.slice_stress()
    T = len(s.type_names)
    tol = 1e-4 if precision == 0 else 1e-9
    assert _close(_sym(got["pair"], T), _sym(ref["pair"], T), tol)
    if s.bond_specs:
        assert _close(got["bond"], ref["bond"], tol)
    if s.bondpair_specs:
        assert _close(got["bondpair"], ref["bondpair"], tol)
    # the profile's zz trace over slices and type pairs is the pair virial's zz
    assert np.abs(got["pair"][..., 8]).sum() > 0


def test_slice_stress_is_the_latest_sample_step(engine_mod, oracle_mod):
    """Sample period 2 over steps 1..3: the profile is step 2's."""
    s = W.bilayer(cells=(10, 10, 10), nlipids=30)
    got = _run(engine_mod, oracle_mod, s, 10, 1, steps=3, period=2)
    o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    o.set_slice_stress(10)
    o.step(1, 2)
    ref = o.slice_stress()
    T = len(s.type_names)
    assert _close(_sym(got["pair"], T), _sym(ref["pair"], T), 1e-9)
    assert _close(got["bond"], ref["bond"], 1e-9)


def test_slice_stress_errors(engine_mod):
    s = W.bilayer(cells=(8, 8, 8), nlipids=16)
    eng = engine_mod.DpdEngine.from_system(s, precision=1)
    with pytest.raises(engine_mod.EngineError):
        eng.slice_stress()                      # off
    with pytest.raises(engine_mod.EngineError):
        eng.set_slice_stress(8, None, 1, None, 0)   # bond types missing for the uploaded bonds
    eng.set_slice_stress_for(s, 8)
    with pytest.raises(engine_mod.EngineError):
        eng.slice_stress()                      # no sample step yet
    eng.step(1, 1)
    assert eng.slice_stress()["pair"].shape == (8, 9, 9)
