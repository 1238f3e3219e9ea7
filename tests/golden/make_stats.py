"""Reference statistics for the thermostat-on validation of the engine.

The oracle in LCG mode follows the reference's trajectory bit for bit
(tests/test_oracle_golden.py), so the statistics below are those of the
reference's own FP64 run at the same dt: instantaneous kT and pressure
(CMonitor::CalculateSingleBeadData, Monitor.cpp:979-982), the radial
distribution function, and for the polymer melt the bond-length and
end-to-end-distance distributions.  Standard errors come from block
averages.  Written to stats_*.npz here:

    python tests/golden/make_stats.py            # 3,000-bead water, 10^3 polymer melt
    python tests/golden/make_stats.py --large    # 12,288-bead water (RDF) and H3T6 bilayer
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from osprey_dpd_b200 import workloads as W  # noqa: E402

RDF_BINS = np.linspace(0.0, 2.5, 51)
BOND_BINS = np.linspace(0.0, 1.2, 49)
E2E_BINS = np.linspace(0.0, 6.0, 31)


def water_system():
    return W.water(10)


def polymer_system():
    return W.polymer_solution(cells=(10, 10, 10), seed=W.BASE_SEED + 40)


def water16_system():
    """12,288-bead water box: the RDF reference at the 1e-3 bound."""
    return W.water(16, seed=W.BASE_SEED + 160)


def bilayer16_system():
    """H3T6 bilayer in water, 16^3 cells (12,288 beads, 376 lipids: the area
    per lipid of the 393,216-bead workload), bonds and tail bond pairs."""
    return W.bilayer(cells=(16, 16, 16), nlipids=376, seed=W.BASE_SEED + 161)


# Bonds of the bilayer: head-tail bead pairs of the linear H3T6 chains.
BILAYER_CHAIN = 9


def rdf_counts(x, L):
    """Pair-distance histogram (minimum image) of one snapshot."""
    from scipy.spatial import cKDTree
    tree = cKDTree(np.mod(x, L), boxsize=L)
    pairs = tree.query_pairs(RDF_BINS[-1], output_type="ndarray")
    d = x[pairs[:, 0]] - x[pairs[:, 1]]
    d -= L * np.round(d / L)
    r = np.sqrt((d * d).sum(axis=1))
    return np.histogram(r, RDF_BINS)[0].astype(np.float64)


def rdf_normalise(counts, nsnap, n, L):
    V = float(np.prod(L))
    shell = 4.0 / 3.0 * np.pi * (RDF_BINS[1:] ** 3 - RDF_BINS[:-1] ** 3)
    ideal = 0.5 * n * (n - 1) / V * shell * nsnap
    return counts / ideal


def chain_stats(u, chain_len, nchains):
    """Bond lengths and end-to-end distances of the linear chains (unPBC)."""
    c = u[: chain_len * nchains].reshape(nchains, chain_len, 3)
    b = np.sqrt(((c[:, 1:] - c[:, :-1]) ** 2).sum(axis=2)).ravel()
    e = np.sqrt(((c[:, -1] - c[:, 0]) ** 2).sum(axis=1))
    return np.histogram(b, BOND_BINS)[0].astype(np.float64), np.histogram(e, E2E_BINS)[0].astype(np.float64)


def bond_lengths(u, head, tail):
    """Histogram of the lengths of the given bonds (unPBC positions, 0-based bead indices)."""
    d = u[head] - u[tail]
    return np.histogram(np.sqrt((d * d).sum(axis=1)), BOND_BINS)[0].astype(np.float64)


def block_se(samples, nblocks=10):
    a = np.asarray(samples, dtype=np.float64)
    m = len(a) // nblocks
    blocks = a[: m * nblocks].reshape(nblocks, m).mean(axis=1)
    return float(blocks.std(ddof=1) / np.sqrt(nblocks))


class Sampler:
    """Accumulates the observables from full bead states."""

    def __init__(self, system, polymer=None):
        self.s = system
        self.L = system.box
        self.kT, self.P = [], []
        self.rdf = np.zeros(len(RDF_BINS) - 1)
        self.bond = np.zeros(len(BOND_BINS) - 1)
        self.e2e = np.zeros(len(E2E_BINS) - 1)
        self.nsnap = 0
        self.polymer = polymer

    def add(self, x, u, v, virial_trace, rdf=True):
        n = self.s.n
        v2 = float((v * v).sum())
        V = float(np.prod(self.L))
        self.kT.append(v2 / (3.0 * n))
        self.P.append(0.3333333333 * (1.0 / V) * (v2 + virial_trace))
        if rdf:
            self.rdf += rdf_counts(x, self.L)
            self.nsnap += 1
        if self.polymer == "bonds":
            self.bond += bond_lengths(u, self.s.bond_head - 1, self.s.bond_tail - 1)
        elif self.polymer:
            b, e = chain_stats(u, *self.polymer)
            self.bond += b
            self.e2e += e

    def result(self):
        out = {"kT_mean": np.mean(self.kT), "kT_se": block_se(self.kT), "P_mean": np.mean(self.P),
               "P_se": block_se(self.P), "nsnap": self.nsnap,
               "rdf": rdf_normalise(self.rdf, self.nsnap, self.s.n, self.L), "rdf_bins": RDF_BINS}
        if self.polymer == "bonds":
            out.update(bond=self.bond / self.bond.sum(), bond_bins=BOND_BINS)
        elif self.polymer:
            out.update(bond=self.bond / self.bond.sum(), bond_bins=BOND_BINS, e2e=self.e2e / self.e2e.sum(),
                       e2e_bins=E2E_BINS)
        return out


def run_oracle(system, equil, steps, every, polymer=None, rdf=True):
    import dpd_oracle
    o = dpd_oracle.Oracle(system, noise=dpd_oracle.NOISE_LCG)
    o.step(1, equil)
    smp = Sampler(system, polymer)
    t = equil + 1
    while t <= equil + steps:
        o.step(t, every)
        t += every
        st = o.state()
        tr = st["stress"].sum(axis=0)
        smp.add(st["x"], st["unpbc"], st["v"], tr[0] + tr[4] + tr[8], rdf=rdf)
    return smp.result()


def large():
    """The 12,288-bead water and bilayer references (several minutes each)."""
    res = run_oracle(water16_system(), 1000, 40000, 10)
    np.savez_compressed(os.path.join(HERE, "stats_water_16.npz"), equil=1000, steps=40000, every=10, **res)
    print("water16", res["kT_mean"], res["kT_se"], res["P_mean"], res["P_se"])
    res = run_oracle(bilayer16_system(), 2000, 20000, 10, polymer="bonds", rdf=False)
    np.savez_compressed(os.path.join(HERE, "stats_bilayer_16.npz"), equil=2000, steps=20000, every=10, **res)
    print("bilayer16", res["kT_mean"], res["kT_se"], res["P_mean"], res["P_se"])


def main():
    res = run_oracle(water_system(), 1000, 20000, 10)
    np.savez_compressed(os.path.join(HERE, "stats_water_10.npz"), equil=1000, steps=20000, every=10, **res)
    print("water", res["kT_mean"], res["kT_se"], res["P_mean"], res["P_se"])
    p = polymer_system()
    nch = p.polymers[0].count
    res = run_oracle(p, 1000, 20000, 10, polymer=(16, nch))
    np.savez_compressed(os.path.join(HERE, "stats_polymer_10.npz"), equil=1000, steps=20000, every=10,
                        nchains=nch, **res)
    print("polymer", res["kT_mean"], res["kT_se"], res["P_mean"], res["P_se"], nch)


if __name__ == "__main__":
    if "--large" in sys.argv:
        large()
    else:
        main()
