"""The half-shell pair schemes (each pair evaluated once, the partner's share
added with atomics; unstaged and staged in shared memory) against the CPU
oracle.  Its force sums are rounded in
a run-dependent order, so the bounds are the tolerances of the full-shell
tests rather than bit equality:
  * mixed precision: forces within 1e-5 of the force RMS after one step,
    1e-4 after five thermostatted steps,
  * FP64: forces within 1e-11 / 1e-10 of the force RMS,
  * the sampled virial (summed over beads) within 2e-5 / 1e-10 of the oracle's,
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


SCHEMES = pytest.mark.parametrize("scheme", [1, 2], ids=["half", "staged"])


def _half(engine_mod, oracle_mod, s, precision, scheme=1, **kw):
    eng = engine_mod.DpdEngine.from_system(s, precision=precision, **kw)
    eng.set_pair_scheme(scheme)
    orc = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX, **kw)
    return eng, orc


@SCHEMES
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_half_shell_one_step(engine_mod, oracle_mod, name, precision, scheme):
    s = SYSTEMS[name]()
    eng, orc = _half(engine_mod, oracle_mod, s, precision, scheme, gamma_scale=0.0)
    eng.step(1, 1)
    orc.step(1, 1)
    g, o = eng.download(), orc.state()
    tol = 1e-5 if precision == 0 else 1e-11
    assert np.array_equal(g["x"], o["x"])
    assert rel_err(g["f"], o["f"]) < tol
    assert np.array_equal(eng.cells(), orc.cells())
    assert eng.status() == 0


@SCHEMES
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_half_shell_thermostat_steps(engine_mod, oracle_mod, name, precision, scheme):
    s = SYSTEMS[name]()
    eng, orc = _half(engine_mod, oracle_mod, s, precision, scheme)
    eng.step(1, 5)
    orc.step(1, 5)
    g, o = eng.download(), orc.state()
    ftol, xtol = (1e-4, 1e-6) if precision == 0 else (1e-10, 1e-12)
    assert rel_err(g["f"], o["f"]) < ftol
    assert float(np.max(np.abs(g["unpbc"] - o["unpbc"]))) < xtol
    assert np.array_equal(eng.cells(), orc.cells())


@SCHEMES
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_half_shell_virial(engine_mod, oracle_mod, precision, scheme):
    s = SYSTEMS["bilayer"]()
    eng, orc = _half(engine_mod, oracle_mod, s, precision, scheme)
    eng.step(1, 3)
    orc.step(1, 3)
    obs = eng.observables()
    vir = orc.state()["stress"].sum(axis=0)
    tol = 2e-5 if precision == 0 else 1e-10
    assert np.allclose(obs["virial"], vir, rtol=0, atol=tol * float(np.max(np.abs(vir))))
    st = eng.download()["stress"].sum(axis=0)
    assert np.allclose(st, vir, rtol=0, atol=tol * float(np.max(np.abs(vir))))


def _dense_cluster_system():
    s = W.water(8)
    rng = np.random.default_rng(7)
    extra = 60
    pts = np.array([3.5, 4.5, 2.5]) + (rng.random((extra, 3)) - 0.5) * 0.9
    return W._assemble("water", s.cells, s.widths, s.density, s.dt, s.lam, s.kT, s.seed, s.type_names, s.a,
                       s.gamma, [W.PolymerSpec("Water", ("W",), s.n + extra)], [], [],
                       np.zeros(s.n + extra, np.int32), np.concatenate([s.unpbc, pts]),
                       np.concatenate([s.v, np.zeros((extra, 3))]))


@pytest.mark.parametrize("tune", ["half=1", "half=1,hitcap=8", "half=1,hitcap=64,bps=1", "half=1,tile=128",
                                  "half=1,tile=128,hitcap=8", "scheme=2", "scheme=2,hitcap=8",
                                  "scheme=2,hitcap=64,bps=1"])
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_half_shell_dense_cell_and_launch_shapes(engine_mod, oracle_mod, precision, tune, monkeypatch):
    """Selected through DPD_TUNE, with a 60-bead cell and extreme hit-list sizes."""
    monkeypatch.setenv("DPD_TUNE", tune)
    s = _dense_cluster_system()
    eng = engine_mod.DpdEngine.from_system(s, precision=precision)
    orc = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    eng.step(1, 2)
    orc.step(1, 2)
    ftol = 1e-4 if precision == 0 else 1e-10
    assert rel_err(eng.download()["f"], orc.state()["f"]) < ftol
    assert eng.status() == 0


@pytest.mark.parametrize("scheme,tile", [(1, 64), (1, 128), (2, 0)], ids=["half", "half_tile128", "staged"])
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_half_shell_replica_batch(engine_mod, oracle_mod, precision, scheme, tile):
    edges, fracs, a_ab, seeds = W.replica_table(4, lo=4, hi=7)
    systems = [W.binary_mixture(n=int(edges[r]), seed=int(seeds[r]), a_ab=float(a_ab[r]), frac_a=float(fracs[r]))
               for r in range(4)]
    batch = engine_mod.DpdBatch(systems, precision=precision)
    batch.set_pair_scheme(scheme)
    batch.set_pair_tile(tile)
    batch.step(1, 3)
    f = batch.split(batch.download()["f"])
    tol = 1e-4 if precision == 0 else 1e-10
    for k, s in enumerate(systems):
        o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
        o.step(1, 3)
        assert rel_err(f[k], o.state()["f"]) < tol
    assert batch.status() == 0


def test_switching_schemes_between_calls(engine_mod):
    """Full -> half -> full on one engine: the captured graphs are rebuilt and
    the trajectory stays within FP64 rounding of a full-shell run."""
    s = SYSTEMS["binary"]()
    a = engine_mod.DpdEngine.from_system(s, precision=1)
    a.step(1, 10)
    b = engine_mod.DpdEngine.from_system(s, precision=1)
    b.step(1, 3)
    b.set_pair_scheme(engine_mod.PAIR_HALF_SHELL)
    b.step(4, 4)
    b.set_pair_scheme(engine_mod.PAIR_FULL_SHELL)
    b.step(8, 3)
    ga, gb = a.download(), b.download()
    assert rel_err(gb["f"], ga["f"]) < 1e-10
    b.set_pair_scheme(engine_mod.PAIR_STAGED)
    b.step(11, 3)
    a.step(11, 3)
    assert rel_err(b.download()["f"], a.download()["f"]) < 1e-10
    with pytest.raises(engine_mod.EngineError):
        b.set_pair_scheme(7)


@pytest.mark.parametrize("scheme", [1, 2], ids=["half", "staged"])
@pytest.mark.parametrize("workload", ["bilayer", "polymer"])
def test_half_shell_matches_full_shell_at_full_size(engine_mod, workload, scheme):
    """The half-shell schemes against the full-shell kernel on the full-size
    workloads (393,216 and 6,291,456 beads), one thermostatted step from the
    same state: the kernels evaluate the same pairs with the same noise, so
    the forces agree to FP32 summation-order rounding."""
    s = W.bilayer() if workload == "bilayer" else W.polymer_solution()
    ref = engine_mod.DpdEngine.from_system(s, precision=0)
    ref.step(1, 1)
    fr = ref.download()["f"]
    ref.close()
    eng = engine_mod.DpdEngine.from_system(s, precision=0)
    eng.set_pair_scheme(scheme)
    eng.step(1, 1)
    fs = eng.download()["f"]
    assert eng.status() == 0
    eng.close()
    assert rel_err(fs, fr) < 2e-5
