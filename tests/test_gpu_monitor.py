"""dpd_engine_monitor (CMonitor::CalculateSingleBeadData / SinglePolymerData /
SingleBondData / SingleBondPairData sums, Monitor.cpp:708-1273, computed on
the device) against a numpy restatement of the same formulas
(oracle/monitor.py): applied to the engine's own downloaded state the two
agree to FP64 summation order (1e-10 relative); applied to the CPU oracle's
state after FP64 steps with the same Philox noise, to 1e-8."""
import os
import sys

import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import monitor as M  # noqa: E402

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "bilayer_htt_phi30": lambda: W.bilayer(cells=(10, 10, 10), nlipids=30, with_htt=True, phi0_deg=30.0),
    "polymer": lambda: W.polymer_solution(cells=(10, 10, 10)),
    "water": lambda: W.water(8),
}
KEYS = ("inertia", "msd", "bond_length", "end_to_end", "bondpair", "mean_bond_length", "mean_sq_bond_length")


def _close(a, b, tol):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-12)
    return a.shape == b.shape and (a.size == 0 or float(np.max(np.abs(a - b))) <= tol * scale)


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_monitor_matches_numpy_on_the_engine_state(engine_mod, name, precision):
    s = SYSTEMS[name]()
    eng = engine_mod.DpdEngine.from_system(s, precision=precision)
    eng.set_monitor_for(s)
    eng.step(1, 5)
    m = eng.monitor()
    g = eng.download()
    ref = M.monitor(s, g["x"], g["unpbc"], s.unpbc, 5, s.dt)
    assert m["step"] == 5 and m["n"] == s.n
    for k in KEYS:
        assert _close(m[k], ref[k], 1e-10), k
    assert np.all(m["msd"] > 0)


def test_monitor_matches_oracle_state(engine_mod, oracle_mod):
    s = SYSTEMS["bilayer_htt_phi30"]()
    eng = engine_mod.DpdEngine.from_system(s, precision=1)
    eng.set_monitor_for(s)
    eng.step(1, 4)
    o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    o.step(1, 4)
    st = o.state()
    ref = M.monitor(s, st["x"], st["unpbc"], s.unpbc, 4, s.dt)
    m = eng.monitor()
    for k in KEYS:
        assert _close(m[k], ref[k], 1e-8), k


def test_monitor_setup_rules(engine_mod):
    s = SYSTEMS["polymer"]()
    eng = engine_mod.DpdEngine.from_system(s, precision=1)
    with pytest.raises(engine_mod.EngineError):
        eng.monitor()                               # not set up
    eng.set_monitor_for(s, initial_unpbc=s.unpbc + 0.25)
    m = eng.monitor()                               # step 0: MSD / N_type only
    assert m["step"] == 0
    assert np.allclose(m["msd"][m["msd"] > 0], 3 * 0.25 ** 2)
    eng.upload_beads(s.ids, s.types, s.movable, s.x, s.unpbc, s.v, s.f)
    with pytest.raises(engine_mod.EngineError):
        eng.monitor()                               # cleared by the upload
