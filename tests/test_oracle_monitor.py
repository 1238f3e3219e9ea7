"""oracle/monitor.py (the numpy restatement of CMonitor's sample data that the
engine's dpd_engine_monitor is checked against) pinned to the reference.

The reference harness runs the unmodified reference on a seeded state with
SamplePeriod = AnalysisPeriod = the run's length, so its analysis file
(dmpcas.<runId>) holds the CMonitor data of one sample -- the last step --
as the reference computes and prints them (CMonitor::CalculateSingleBeadData /
SinglePolymerData / SingleBondData / SingleBondPairData, Monitor.cpp:708-1273):
the inertia tensor, the mean bond length overall and per bond type, the
mean end-to-end distance per polymer type, and per bond-pair type P2, the
mean first and second bond lengths and <dphi^2>/<dphi>^2; its history file
(dmpchs.<runId>) adds the MSD of every bead type.  The restatement,
applied to the reference's own final state (dumped by the harness), must give
the same numbers to the file's printed precision (6 significant digits:
relative 1e-5 of each block's largest entry).  Temperature and pressure are
checked the same way from the dumped velocities and per-bead stress."""
import os
import shutil
import sys
import tempfile

import numpy as np
import pytest

from conftest import ROOT
from osprey_dpd_b200 import workloads as W

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import monitor as M  # noqa: E402

SYSTEMS = {
    "bilayer_htt_phi30": lambda: W.bilayer(cells=(10, 10, 10), nlipids=30, with_htt=True, phi0_deg=30.0),
    "bilayer": lambda: W.bilayer(cells=(12, 12, 12), nlipids=60),
    "polymer": lambda: W.polymer_solution(cells=(10, 10, 10)),
    "water": lambda: W.water(8),
}
STEPS = 5


def parse_analysis(path):
    """dmpcas blocks: a title line, then rows of numbers (means, then SDs)."""
    blocks, title, rows = {}, None, []
    for ln in open(path):
        s = ln.strip()
        if not s:
            if title is not None:
                blocks[title] = np.array(rows)
            title, rows = None, []
            continue
        try:
            vals = [float(v) for v in s.split()]
        except ValueError:
            if title is not None:
                blocks[title] = np.array(rows)
            title, rows = s, []
            continue
        rows.append(vals)
    if title is not None:
        blocks[title] = np.array(rows)
    return blocks


def _close(a, b, rel=1e-5):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) <= rel * scale


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_monitor_restatement_equals_the_reference_sample(oracle_mod, name):
    if not os.path.exists(oracle_mod.REF_DRIVER):
        pytest.skip("reference harness not built here")
    s = SYSTEMS[name]()
    wd = tempfile.mkdtemp(prefix="dpdmon_")
    try:
        _, dump, _ = oracle_mod.run_reference(s, STEPS, workdir=wd)
        ref = parse_analysis(os.path.join(wd, "dmpcas.r"))
        hist = [list(map(float, ln.split())) for ln in open(os.path.join(wd, "dmpchs.r")) if ln.strip()][-1]
    finally:
        shutil.rmtree(wd, ignore_errors=True)
    got = M.monitor(s, dump["x"], dump["unpbc"], s.unpbc, STEPS, s.dt)
    # inertia tensor (means in the first three columns)
    assert _close(got["inertia"], ref["Inertia"][:, :3])
    # temperature and pressure from the dumped state (Monitor.cpp:979-982)
    v2 = float((dump["v"] ** 2).sum())
    tr = dump["stress"].sum(axis=0)
    V = float(np.prod(s.box))
    assert _close(v2 / (3.0 * s.n), ref["Temperature"][0, 0])
    assert _close(0.3333333333 / V * (v2 + tr[0] + tr[4] + tr[8]), ref["Pressure"][0, 0])
    # bonds: overall mean and per bond type, named by its head and tail bead types
    if len(s.bond_specs):
        assert _close(got["mean_bond_length"], ref["Bond Length"][0, 0])
        for k, b in enumerate(s.bond_specs):
            assert _close(got["bond_length"][k], ref[f"{b.name1}{b.name2} bond length"][0, 0]), b
    # the history row of the sample (CMonitor::SaveHistoryState, Monitor.cpp:1760-1806): time, kT, P,
    # three energy terms, then the MSD of every bead type and the end-to-end distance of every polymer type
    T = len(s.type_names)
    assert hist[0] == STEPS
    assert _close(hist[6:6 + T], got["msd"])
    assert _close(hist[6 + T:6 + T + len(s.polymers)], got["end_to_end"]) or not np.any(got["end_to_end"])
    # polymers: mean end-to-end distance per polymer type
    for k, p in enumerate(s.polymers):
        assert _close(got["end_to_end"][k], ref[f"{p.name} EE distance"][0, 0]), p.name
    # bond pairs per type: P2, first and second bond length, <dphi^2>/<dphi>^2
    for k, bp in enumerate(s.bondpair_specs):
        nm = f"{bp.name1}{bp.name2}{bp.name3}"
        for col, title in ((0, "P2(x)"), (1, "first bond length"), (2, "second bond length"),
                           (5, "<phi**2>/<phi>**2")):
            assert _close(got["bondpair"][k, col], ref[f"{nm} {title}"][0, 0]), (nm, title)
