"""Loader of the restart golden fixtures (tests/golden/restart_*.npz)."""
import os

import numpy as np

from osprey_dpd_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = {
    "restart_bilayer_6": lambda: W.bilayer(cells=(6, 6, 6), nlipids=8),
    "restart_polymer_6": lambda: W.polymer_solution(cells=(6, 6, 6)),
}


def load_case(name):
    """(system carrying the reference's state after the run, fixture dict)."""
    s = CASES[name]()
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    g = {k: z[k] for k in ("x", "unpbc", "v", "f")}
    g["restart"] = z["restart"].tobytes()
    g["steps"] = int(z["steps"])
    s = s.copy()
    s.x, s.unpbc, s.v, s.f = g["x"].copy(), g["unpbc"].copy(), g["v"].copy(), g["f"].copy()
    return s, g
