"""Generates lamella_*.npz here: the initial state the unmodified reference
(oracle/_ref/osprey_ref_driver --dump-initial) builds for a control file with
`State lamella` (CLamellaBuilder::Assemble, LamellaBuilder.cpp:126-1010):
bead creation order (ids, types), the polymers (first bead, type), the bonds
in the reference's polymer order (bead indices), the generator seed
(|RNGSeed|), box lengths, kT and the lamella parameters.

    python tests/golden/make_lamella_golden.py
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


def layout(system):
    first, ptype = [0], []
    for t, p in enumerate(system.polymers):
        for _ in range(p.count):
            first.append(first[-1] + len(p.beads))
            ptype.append(t)
    return np.array(first, np.int64), np.array(ptype, np.int32)


def record(system, normal, linearise, upper_fraction):
    nv = [0, 0, 0]
    nv[normal] = 1
    block = W.lamella_block("Lipid", normal=tuple(nv), centre=0.5, thickness=5.0, linearise=linearise,
                            upper_fraction=upper_fraction)
    summ, _, topo = O.run_reference(system, 1, inject=False, dump=False, topology=True, initial=True, state=block)
    ini = summ["initial"]
    if not np.array_equal(ini["id"], np.arange(1, system.n + 1)):
        raise RuntimeError("unexpected bead id order")
    first, ptype = layout(system)
    return dict(ids=ini["id"], types=ini["type"].astype(np.int32), x=ini["x"], unpbc=ini["unpbc"], v=ini["v"],
                poly_first=first, poly_type=ptype, bond_head=topo["bond_head"] - 1, bond_tail=topo["bond_tail"] - 1,
                seed=np.uint64(abs(-abs(int(system.seed)) % 2147483647)), L=np.asarray(system.box, np.float64),
                kT=np.float64(system.kT), lipid_type=np.int32(0), head_offset=np.int32(0),
                tail_offset=np.int32(len(system.polymers[0].beads) - 1), normal=np.int32(normal),
                centre=np.float64(0.5), thickness=np.float64(5.0), linearise=np.int32(int(linearise)),
                upper_fraction=np.float64(upper_fraction))


def main():
    cases = {
        "lamella_z_straight": (W.bilayer(cells=(10, 10, 10), nlipids=60), 2, True, 0.5),
        "lamella_x_straight": (W.bilayer(cells=(12, 8, 8), nlipids=60), 0, True, 0.5),
        "lamella_y_scattered": (W.bilayer(cells=(8, 12, 8), nlipids=60), 1, False, 0.5),
        "lamella_z_upper_only": (W.bilayer(cells=(8, 8, 12), nlipids=50), 2, False, 1.0),
    }
    for name, (system, normal, linearise, uf) in cases.items():
        rec = record(system, normal, linearise, uf)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
        print(name, system.n, len(rec["bond_head"]))


if __name__ == "__main__":
    main()
