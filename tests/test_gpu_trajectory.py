"""1,000-step deterministic trajectories (sigma = 0) against the oracle.

A DPD fluid is chaotic: any difference in the last bit grows exponentially,
so the stated tolerance is the oracle's own sensitivity.  At each checkpoint
the engine's distance from the oracle (max |unPBC difference| over beads) must
stay within 10x the distance between two oracle runs whose initial states
differ by eps in one coordinate, eps being the precision of the engine's
forces (1e-13 for FP64, 1e-6 for the FP32 forces of mixed mode), plus 1e-11.
Both sigma = 0 variants of the reference are covered: kT = 0 (dissipative
forces kept, CNTCell.cpp:190) and gamma = 0 (ToggleDPDBeadThermostat)."""
import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.gpu

CHECKPOINTS = (100, 250, 500, 1000)


@pytest.mark.parametrize("variant", ["kT0", "gamma0"])
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_sigma0_trajectory_within_chaos_envelope(engine_mod, oracle_mod, precision, variant):
    s = W.water(8)
    kw = {"kT": 0.0} if variant == "kT0" else {"gamma_scale": 0.0}
    eps = 1e-6 if precision == 0 else 1e-13
    s_pert = s.copy()
    s_pert.x[0, 0] += eps
    s_pert.unpbc[0, 0] += eps
    eng = engine_mod.DpdEngine.from_system(s, precision=precision, **kw)
    orc = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX, **kw)
    pert = oracle_mod.Oracle(s_pert, noise=oracle_mod.NOISE_PHILOX, **kw)
    t = 1
    report = []
    for cp in CHECKPOINTS:
        n = cp - t + 1
        eng.step(t, n)
        orc.step(t, n)
        pert.step(t, n)
        t = cp + 1
        g, o, p = eng.download()["unpbc"], orc.state()["unpbc"], pert.state()["unpbc"]
        d_gpu = float(np.max(np.abs(g - o)))
        d_env = float(np.max(np.abs(p - o)))
        report.append((cp, d_gpu, d_env))
        assert d_gpu <= 10.0 * d_env + 1e-11, report
    print("\n", variant, precision, report)
