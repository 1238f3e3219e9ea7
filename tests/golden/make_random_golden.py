"""Generates random_*.npz here: the initial state the unmodified reference
(oracle/_ref/osprey_ref_driver --dump-initial) builds for a control file with
`State random` (CRandomBuilder::Assemble, RandomBuilder.cpp:71-361), with the
bead creation order (ids, types), the bonds in the reference's polymer order
(as bead indices), the generator seed (|RNGSeed|), box lengths and kT.

    python tests/golden/make_random_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from osprey_dpd_b200 import workloads as W  # noqa: E402
import dpd_oracle as O  # noqa: E402


def control_seed(system) -> int:
    # write_dmpci writes RNGSeed as -|seed| mod 2^31-1; CCNTCell::SetRNGSeed takes its magnitude
    return abs(-abs(int(system.seed)) % 2147483647)


def record(system):
    summ, _, topo = O.run_reference(system, 1, inject=False, dump=False, topology=True, initial=True)
    ini = summ["initial"]
    if not np.array_equal(ini["id"], np.arange(1, system.n + 1)):
        raise RuntimeError("unexpected bead id order")
    return dict(ids=ini["id"], types=ini["type"].astype(np.int32), x=ini["x"], unpbc=ini["unpbc"], v=ini["v"],
                bond_head=topo["bond_head"] - 1, bond_tail=topo["bond_tail"] - 1, seed=np.uint64(control_seed(system)),
                L=np.asarray(system.box, dtype=np.float64), kT=np.float64(system.kT))


def main():
    cases = {
        "random_water_10": W.water(n=10),
        "random_polymer_8": W.polymer_solution(cells=(8, 8, 8)),
    }
    for name, system in cases.items():
        rec = record(system)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
        print(name, system.n, len(rec["bond_head"]))


if __name__ == "__main__":
    main()
