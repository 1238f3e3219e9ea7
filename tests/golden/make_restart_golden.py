"""Generates restart_*.npz here: the restart file the unmodified reference
(oracle/_ref/osprey_ref_driver) writes at the end of a short run
(CRestartState::Serialize, RestartState.cpp:100-163), together with its
full-precision state at that step (the harness dump), so a writer given the
same state can be compared byte for byte.

    python tests/golden/make_restart_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from osprey_dpd_b200 import workloads as W  # noqa: E402


def cases():
    return {
        "restart_bilayer_6": (lambda: W.bilayer(cells=(6, 6, 6), nlipids=8), 3),
        "restart_polymer_6": (lambda: W.polymer_solution(cells=(6, 6, 6)), 3),
    }


def main():
    import dpd_oracle
    for name, (make, steps) in cases().items():
        s = make()
        wd = tempfile.mkdtemp(prefix="dpdrs_")
        summary, d, _ = dpd_oracle.run_reference(s, steps, workdir=wd, rng_seed=s.seed)
        with open(os.path.join(wd, f"dmpcrs.r.con.{steps}.dat"), "rb") as fh:
            text = fh.read()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), steps=steps, x=d["x"], unpbc=d["unpbc"],
                            v=d["v"], f=d["f"], restart=np.frombuffer(text, dtype=np.uint8))
        print(name, summary, len(text), "bytes")


if __name__ == "__main__":
    main()
