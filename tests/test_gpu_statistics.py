"""Thermostat-on validation against the reference's own statistics.

With the thermostat on, no parallel evaluation can follow the reference's
serial pair-noise stream, so the engine is validated statistically: the same
systems, the same dt and protocol (1,000 steps to equilibrate, then 20,000
steps sampled every 10), compared with tests/golden/stats_*.npz, which holds
the statistics of the reference's trajectory (tests/golden/make_stats.py).

Bounds stated here:
  * mean kT within 0.5 % of the reference's;
  * mean pressure within 0.5 % and within 5 combined standard errors;
  * RDF (3,000-bead water, 20,000 steps): root-mean-square difference over
    0.25 <= r < 2.5 below 2e-3 (the two finite samples alone give about 1e-3);
  * RDF at the 1e-3 bound ("RDF L2 error": the root-mean-square difference
    over the bins 0.25 <= r < 2.5, width 0.05): 12,288-bead water, 40,000
    steps sampled every 10 on both sides, below 1e-3;
  * polymer bond-length and end-to-end distributions: total-variation
    distance below 0.01 and 0.08;
  * H3T6 bilayer in water (12,288 beads, bonds and tail bond pairs): kT and
    pressure as above, bond-length distribution total-variation distance
    below 0.01.
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


def _rdf_counts_gpu(x, L, torch, chunk=6144):
    """Pair-distance histogram (minimum image, each unordered pair once) of one
    snapshot on the GPU, in the bins of the reference statistics."""
    dev = torch.device("cuda", 0)
    X = torch.as_tensor(np.mod(x, L), dtype=torch.float64, device=dev)
    Lt = torch.as_tensor(L, dtype=torch.float64, device=dev)
    edges = torch.as_tensor(MS.RDF_BINS, dtype=torch.float64, device=dev)
    counts = torch.zeros(len(MS.RDF_BINS) - 1, dtype=torch.float64, device=dev)
    n = X.shape[0]
    for a in range(0, n, chunk):
        d = X[a:a + chunk, None, :] - X[None, :, :]
        d -= Lt * torch.round(d / Lt)
        r = torch.sqrt((d * d).sum(dim=2))
        ii = torch.arange(a, min(a + chunk, n), device=dev)[:, None]
        jj = torch.arange(n, device=dev)[None, :]
        r = r[(jj > ii) & (r < MS.RDF_BINS[-1])]
        idx = torch.bucketize(r, edges, right=True) - 1
        counts += torch.bincount(idx, minlength=len(MS.RDF_BINS) - 1)[: len(MS.RDF_BINS) - 1].double()
    return counts.cpu().numpy()


def _run_engine_large(engine_mod, system, precision, ref, bonds=False, rdf=True):
    """The fixture's protocol on the engine: equilibrate, then sample every
    `every` steps (kT, P, and the RDF or the bond lengths)."""
    import torch
    eng = engine_mod.DpdEngine.from_system(system, precision=precision, device=0)
    every = int(ref["every"])
    eng.set_sample_period(every)
    equil, steps = int(ref["equil"]), int(ref["steps"])
    eng.step(1, equil)
    kT, P = [], []
    rdf_counts = np.zeros(len(MS.RDF_BINS) - 1)
    bond = np.zeros(len(MS.BOND_BINS) - 1)
    nsnap = 0
    V = float(np.prod(system.box))
    t = equil + 1
    while t <= equil + steps:
        eng.step(t, every)
        t += every
        st = eng.download(stress=False)
        vir = eng.observables()["virial"]
        v2 = float((st["v"] ** 2).sum())
        kT.append(v2 / (3.0 * system.n))
        P.append(0.3333333333 * (1.0 / V) * (v2 + vir[0] + vir[4] + vir[8]))
        if rdf:
            rdf_counts += _rdf_counts_gpu(st["x"], system.box, torch)
            nsnap += 1
        if bonds:
            bond += MS.bond_lengths(st["unpbc"], system.bond_head - 1, system.bond_tail - 1)
    assert eng.status() & ~engine_mod.STATUS_CELL_SKIP == 0
    eng.close()
    out = {"kT_mean": np.mean(kT), "kT_se": MS.block_se(kT), "P_mean": np.mean(P), "P_se": MS.block_se(P)}
    if rdf:
        out["rdf"] = MS.rdf_normalise(rdf_counts, nsnap, system.n, system.box)
    if bonds:
        out["bond"] = bond / bond.sum()
    return out


def _check_kT_P(got, ref):
    assert abs(got["kT_mean"] - ref["kT_mean"]) < 0.005 * ref["kT_mean"]
    se = np.hypot(got["P_se"], float(ref["P_se"]))
    assert abs(got["P_mean"] - ref["P_mean"]) < min(0.005 * ref["P_mean"], max(5 * se, 0.02))


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


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_water_rdf_at_the_1e3_bound(engine_mod, precision):
    """12,288-bead water: RDF L2 error (RMS over the bins) below 1e-3."""
    ref = np.load(os.path.join(GOLDEN, "stats_water_16.npz"))
    got = _run_engine_large(engine_mod, MS.water16_system(), precision, ref)
    err = _rdf_rms(got["rdf"], ref["rdf"])
    print(f"\nwater16[{precision}] kT {got['kT_mean']:.5f} vs {float(ref['kT_mean']):.5f}, "
          f"P {got['P_mean']:.4f} vs {float(ref['P_mean']):.4f}, rdf L2 {err:.2e}")
    _check_kT_P(got, ref)
    assert err < 1e-3


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_bilayer_kT_pressure_and_bond_lengths(engine_mod, precision):
    """H3T6 bilayer in water (bonds, tail bond pairs): kT, P and the bond-length
    distribution against the reference's trajectory."""
    ref = np.load(os.path.join(GOLDEN, "stats_bilayer_16.npz"))
    got = _run_engine_large(engine_mod, MS.bilayer16_system(), precision, ref, bonds=True, rdf=False)
    tv = 0.5 * float(np.abs(got["bond"] - ref["bond"]).sum())
    print(f"\nbilayer16[{precision}] kT {got['kT_mean']:.5f} vs {float(ref['kT_mean']):.5f}, "
          f"P {got['P_mean']:.4f} vs {float(ref['P_mean']):.4f} (se {got['P_se']:.4f}/{float(ref['P_se']):.4f}), "
          f"bond TV {tv:.4f}")
    _check_kT_P(got, ref)
    assert tv < 0.01
