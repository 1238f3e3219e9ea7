"""Generates the golden fixtures in this directory by running the unmodified
Osprey-DPD reference (oracle/_ref/osprey_ref_driver, built by
`make -C oracle ref` from the reference sources) on small seeded systems.

Each case stores the reference's state after `steps` steps (x, unPBC, v, F
for every bead, the summed per-bead stress) and a checksum of the generated
input, so a change in the input generator is reported as such.  The pair
noise LCG is restarted at the system seed before the step loop
(`--rng-seed`), which makes the run reproducible from the fixture alone.

    python tests/golden/make_golden.py          # rewrites *.npz here
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from osprey_dpd_b200 import workloads as W  # noqa: E402


def cases():
    """name -> (system factory, steps, kT override, gamma scale)."""
    return {
        "water_6": (lambda: W.water(6), 25, None, 1.0),
        "water_6_kT0": (lambda: W.water(6), 25, 0.0, 1.0),
        "water_6_gamma0": (lambda: W.water(6), 25, None, 0.0),
        "binary_6x6x7": (lambda: W.binary_mixture(cells=(6, 6, 7)), 25, None, 1.0),
        "bilayer_7": (lambda: W.bilayer(cells=(7, 7, 7), nlipids=12), 25, None, 1.0),
        "polymer_7": (lambda: W.polymer_solution(cells=(7, 7, 7)), 25, None, 1.0),
    }


def input_checksum(s) -> str:
    h = hashlib.sha256()
    for a in (s.ids, s.types, s.x, s.unpbc, s.v, s.bond_head, s.bond_tail, s.angle_first, s.angle_second):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    import dpd_oracle
    for name, (make, steps, kT, gs) in cases().items():
        s = make()
        summary, d, topo = dpd_oracle.run_reference(s, steps, kT=kT, gamma_scale=gs, topology=True,
                                                     rng_seed=s.seed)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            steps=steps, kT=-1.0 if kT is None else kT, gamma_scale=gs, checksum=input_checksum(s),
            x=d["x"], unpbc=d["unpbc"], v=d["v"], f=d["f"], stress_sum=d["stress"].sum(axis=0),
            stress_first=d["stress"][:8],
            bond_head=topo["bond_head"], bond_tail=topo["bond_tail"],
            angle_first=topo["angle_first"], angle_second=topo["angle_second"])
        print(name, summary)


if __name__ == "__main__":
    main()
