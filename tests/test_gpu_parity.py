"""Parity of the CUDA engine (through its C ABI) with the CPU oracle.

The oracle is the reference's algorithm restated in C and pinned bit-for-bit
against the reference binary (tests/test_oracle_reference.py,
tests/test_oracle_golden.py).  Tolerances, stated per test:
  * mixed precision (FP32 forces): forces within 1e-5 of the force RMS,
  * FP64: forces within 1e-11 of the force RMS,
  * positions after the first step: bit-identical (same FP64 drift),
  * CNT cell assignment: identical.
"""
import numpy as np
import pytest

from conftest import rel_err
from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "water": lambda: W.water(10),
    "binary": lambda: W.binary_mixture(cells=(8, 9, 10)),
    "bilayer": lambda: W.bilayer(cells=(12, 12, 12), nlipids=60),
    "polymer": lambda: W.polymer_solution(cells=(12, 12, 12)),
}
FORCE_TOL = {0: 1e-5, 1: 1e-11}


def _pair(engine_mod, oracle_mod, system, precision, noise=None, **kw):
    noise = oracle_mod.NOISE_PHILOX if noise is None else noise
    eng = engine_mod.DpdEngine.from_system(system, precision=precision, **kw)
    orc = oracle_mod.Oracle(system, noise=noise, **kw)
    return eng, orc


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_one_step_conservative_and_bonded(engine_mod, oracle_mod, name, precision):
    """Thermostat off (gamma = 0): conservative, bond and bond-pair forces."""
    s = SYSTEMS[name]()
    eng, orc = _pair(engine_mod, oracle_mod, s, precision, gamma_scale=0.0)
    eng.step(1, 1)
    orc.step(1, 1)
    g, o = eng.download(), orc.state()
    assert np.array_equal(g["x"], o["x"]), "first-step drift must be bit-identical"
    assert rel_err(g["f"], o["f"]) < FORCE_TOL[precision]
    assert rel_err(g["v"], o["v"], scale=1.0) < FORCE_TOL[precision]
    assert np.allclose(g["unpbc"], o["unpbc"], rtol=0, atol=1e-12)
    assert np.array_equal(eng.cells(), orc.cells())
    assert eng.status() == 0


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
@pytest.mark.parametrize("name", ["water", "bilayer"])
def test_one_step_dissipative(engine_mod, oracle_mod, name, precision):
    """kT = 0: conservative + dissipative forces, no noise (CNTCell.cpp:190)."""
    s = SYSTEMS[name]()
    eng, orc = _pair(engine_mod, oracle_mod, s, precision, kT=0.0)
    eng.step(1, 1)
    orc.step(1, 1)
    g, o = eng.download(), orc.state()
    assert rel_err(g["f"], o["f"]) < FORCE_TOL[precision]


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_thermostat_philox_steps(engine_mod, oracle_mod, name, precision):
    """Thermostat on with the shared Philox pair noise: 5 steps agree to
    1e-4 (mixed) / 1e-10 (FP64) of the force RMS, positions to 1e-6 / 1e-12."""
    s = SYSTEMS[name]()
    eng, orc = _pair(engine_mod, oracle_mod, s, precision)
    eng.step(1, 5)
    orc.step(1, 5)
    g, o = eng.download(), orc.state()
    ftol, xtol = (1e-4, 1e-6) if precision == 0 else (1e-10, 1e-12)
    assert rel_err(g["f"], o["f"]) < ftol
    assert float(np.max(np.abs(g["unpbc"] - o["unpbc"]))) < xtol
    assert np.array_equal(eng.cells(), orc.cells())


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_observables_match_oracle(engine_mod, oracle_mod, precision):
    s = SYSTEMS["bilayer"]()
    eng, orc = _pair(engine_mod, oracle_mod, s, precision)
    eng.step(1, 3)
    orc.step(1, 3)
    obs = eng.observables()
    o = orc.state()
    v2 = float(np.sum(o["v"] ** 2))
    vir = o["stress"].sum(axis=0)
    V = float(np.prod(s.box))
    tol = 2e-5 if precision == 0 else 1e-10
    assert obs["has_virial"]
    assert abs(obs["kT"] - v2 / (3 * s.n)) < tol * (v2 / (3 * s.n))
    assert np.allclose(obs["virial"], vir, rtol=0, atol=tol * float(np.max(np.abs(vir))))
    p_ref = 0.3333333333 * (1.0 / V) * (v2 + vir[0] + vir[4] + vir[8])
    assert abs(obs["pressure"] - p_ref) < tol * abs(p_ref)
    # the FP64 reduction itself is exact to ~1e-12; total momentum moves by the
    # FP32 rounding of the per-bead force sums in mixed mode (~sqrt(N) * 1e-6 per step)
    g = eng.download()
    assert np.allclose(obs["sum_v"], g["v"].sum(axis=0), rtol=0, atol=1e-10)
    drift = 1e-4 if precision == 0 else 1e-10
    assert np.allclose(obs["sum_v"], o["v"].sum(axis=0), rtol=0, atol=drift)


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_bitwise_deterministic(engine_mod, precision):
    s = SYSTEMS["bilayer"]()
    outs = []
    for _ in range(2):
        eng = engine_mod.DpdEngine.from_system(s, precision=precision)
        eng.step(1, 20)
        outs.append(eng.download())
        eng.close()
    for k in ("x", "v", "f", "stress"):
        assert np.array_equal(outs[0][k], outs[1][k]), k


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_sample_period_takes_sums_at_sample_steps(engine_mod, oracle_mod, precision):
    """With a sample period the sums describe the latest step t with
    t % period == 0 (ISimState::TimeToSample), not the last step run."""
    s = SYSTEMS["bilayer"]()
    eng, orc = _pair(engine_mod, oracle_mod, s, precision)
    eng.set_sample_period(4)
    eng.step(1, 6)
    obs = eng.observables()
    assert obs["step"] == 4 and obs["has_virial"]
    orc.step(1, 4)
    o = orc.state()
    v2 = float(np.sum(o["v"] ** 2))
    tol = 2e-5 if precision == 0 else 1e-10
    assert abs(obs["kT"] - v2 / (3 * s.n)) < tol * (v2 / (3 * s.n))
    vir = o["stress"].sum(axis=0)
    assert np.allclose(obs["virial"], vir, rtol=0, atol=tol * float(np.max(np.abs(vir))))


def _dense_cluster_system():
    """Water with 60 extra beads packed inside one cell: neighbour rows far
    longer than any per-lane hit list, and many overlapping pairs."""
    s = W.water(8)
    rng = np.random.default_rng(7)
    extra = 60
    c = np.array([3.5, 4.5, 2.5])
    pts = c + (rng.random((extra, 3)) - 0.5) * 0.9
    s2 = W._assemble("water", s.cells, s.widths, s.density, s.dt, s.lam, s.kT, s.seed, s.type_names, s.a,
                     s.gamma, [W.PolymerSpec("Water", ("W",), s.n + extra)], [], [],
                     np.zeros(s.n + extra, np.int32), np.concatenate([s.unpbc, pts]),
                     np.concatenate([s.v, np.zeros((extra, 3))]))
    return s2


@pytest.mark.parametrize("tune", ["", "hitcap=8", "hitcap=64,bps=1"])
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_dense_cell_and_launch_shapes(engine_mod, oracle_mod, precision, tune, monkeypatch):
    """A cell with 60+ beads, under the default and extreme pair-kernel
    launch shapes (DPD_TUNE): forces still match the oracle."""
    monkeypatch.setenv("DPD_TUNE", tune)
    s = _dense_cluster_system()
    eng, orc = _pair(engine_mod, oracle_mod, s, precision)
    eng.step(1, 2)
    orc.step(1, 2)
    g, o = eng.download(), orc.state()
    ftol = 1e-4 if precision == 0 else 1e-10
    assert rel_err(g["f"], o["f"]) < ftol
    assert eng.status() == 0


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_graph_replay_equals_direct_launches(engine_mod, precision, monkeypatch):
    """Multi-step calls replay a captured CUDA graph; results are identical to
    launching the kernels one by one (DPD_GRAPHS=0)."""
    s = SYSTEMS["bilayer"]()
    outs = []
    for graphs in ("1", "0"):
        monkeypatch.setenv("DPD_GRAPHS", graphs)
        eng = engine_mod.DpdEngine.from_system(s, precision=precision)
        eng.set_sample_period(5)
        eng.step(1, 7)       # odd count: the buffer parity flips
        eng.step(8, 7)
        eng.step(15, 10)
        outs.append((eng.download(), eng.observables(), eng.launch_count()))
        eng.close()
    for k in ("x", "v", "f", "stress"):
        assert np.array_equal(outs[0][0][k], outs[1][0][k]), k
    assert outs[0][1] == outs[1][1]
    assert outs[0][2] == outs[1][2]
