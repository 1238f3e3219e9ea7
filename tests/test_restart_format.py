"""The restart-file format the engine writes (dpd_engine_write_restart), as a
plain restatement of CRestartState::Serialize (RestartState.cpp:100-163):
given the reference's own full-precision state, "%.6g" fields reproduce the
bead section of the file the reference wrote byte for byte (golden fixtures made by
tests/golden/make_restart_golden.py).  CPU only: this pins the format the
CUDA library's writer uses; test_gpu_restart.py checks the writer itself."""
import os

import numpy as np
import pytest

from osprey_dpd_b200 import engine as E, workloads as W
from golden_restart import CASES, load_case

HERE = os.path.dirname(os.path.abspath(__file__))


def format_restart(system, x, unpbc, v, f, radius=0.5):
    order, pid, pty = E.restart_layout(system)
    L = system.box
    x = x.copy()
    for d in range(3):   # CheckBeadWithinBox, RestartState.cpp:488-530
        c = x[:, d]
        c[(c > L[d] - 0.001) | (c < 0.001)] = 0.001
    lines = ["0 0 0"]
    for k in order:
        vals = [radius, *x[k], *unpbc[k], *v[k], *f[k]]
        lines.append(f"{pid[k]} {pty[k]} {system.ids[k]} {system.types[k]} " + " ".join("%.6g" % q for q in vals))
    return ("\n".join(lines) + "\n").encode()


def bead_section(restart: bytes) -> bytes:
    """The part CRestartState::Serialize writes: everything before the
    "inclusive" appendix that CInclusiveRestartState adds from the reference's
    own type tables and command targets (InclusiveRestartState.cpp:190-205)."""
    k = restart.find(b"inclusive\n")
    return restart if k < 0 else restart[:k]


@pytest.mark.parametrize("name", list(CASES))
def test_restart_format_matches_reference_file(name):
    s, g = load_case(name)
    sec = bead_section(g["restart"])
    assert sec.count(b"\n") == s.n + 1
    assert format_restart(s, g["x"], g["unpbc"], g["v"], g["f"]) == sec
