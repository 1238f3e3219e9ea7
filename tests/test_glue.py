"""The reference-side binding end to end: the reference's own program with
the engine in CSimBox::Evolve (osprey_dpd_b200/glue: the OSPREY_DPD_CUDA copy
of SimBox.cpp, the binding, the engine library), run on control files in the
reference's dmpci format (tests/golden/dmpci), compared with the reference
program's own runs of the same files (tests/golden/glue_*.npz, made by
tests/golden/make_glue_golden.py).

Bounds: the mean temperature and pressure that CMonitor writes to the history
file over the second analysis period (after equilibration) agree with the
reference's within 5 combined block standard errors and within 1 % -- the
thermostat noise differs (counter-based pairs on the device, the serial LCG
in the reference), so the comparison is statistical.  Error path: a bead
state made non-finite on the host stops the run through the reference's own
CLogSimErrorTrace + ccStopNoSave, for an upload the engine rejects and for a
state that turns non-finite on the device.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, gpu_available

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_glue_golden as G  # noqa: E402

GLUE = os.path.join(ROOT, "osprey_dpd_b200", "_build", "glue", "osprey_dpd_cuda")


def _glue_binary():
    if not os.path.exists(GLUE):
        raise FileNotFoundError(f"{GLUE} is missing: run `make -C osprey_dpd_b200/glue` where the reference "
                                f"sources are present")
    return GLUE


def _block_se(a, nblocks=10):
    m = len(a) // nblocks
    b = np.asarray(a[: m * nblocks]).reshape(nblocks, m).mean(axis=1)
    return float(b.std(ddof=1) / np.sqrt(nblocks))


def _compare(name, t_from):
    ref = np.load(os.path.join(ROOT, "tests", "golden", f"glue_{name}.npz"))["history"]
    got, log, seconds = G.run(_glue_binary(), name)
    assert "error" not in log.lower(), log[-2000:]
    assert got.shape[0] == ref.shape[0] and np.array_equal(got[:, 0], ref[:, 0])
    for col, what in ((1, "temperature"), (2, "pressure")):
        r = ref[ref[:, 0] > t_from, col]
        g = got[got[:, 0] > t_from, col]
        se = np.hypot(_block_se(r), _block_se(g))
        print(f"\n{name} {what}: engine {g.mean():.5f} +- {_block_se(g):.5f}, reference {r.mean():.5f} "
              f"+- {_block_se(r):.5f} ({seconds:.1f} s)")
        assert abs(g.mean() - r.mean()) < 5 * se
        assert abs(g.mean() - r.mean()) < 0.01 * abs(r.mean())


@pytest.mark.skipif(gpu_available(), reason="checks the error path when no CUDA device exists")
def test_binding_stops_the_run_when_the_engine_cannot_start():
    if not os.path.exists(GLUE):
        pytest.skip("binding not built here (needs the reference sources)")
    _, log, _ = G.run(GLUE, "water")
    assert "B200 engine: dpd_engine_create failed" in log
    assert "stopped without save at time 2" in log


@pytest.mark.gpu
def test_binding_runs_the_water_control_file():
    _compare("water", 5000)


@pytest.mark.gpu
def test_binding_runs_the_bilayer_control_file_with_a_time_step_change():
    _compare("bilayer", 10000)


@pytest.mark.gpu
def test_binding_stops_the_run_on_a_state_that_turns_nonfinite():
    """A 1e308 force on one uploaded bead: the first step makes the state
    non-finite on the device; a later dpd_engine_step returns DPD_E_STATUS
    and the binding stops the run through the reference's error path."""
    _, log, _ = G.run(_glue_binary(), "water", env={"OSPREY_DPD_GLUE_INJECT": "force:17"})
    assert "B200 engine: step failed (-5)" in log and "non-finite" in log
    assert "stopped without save" in log


@pytest.mark.gpu
def test_binding_stops_the_run_on_a_nonfinite_upload():
    _, log, _ = G.run(_glue_binary(), "water", env={"OSPREY_DPD_GLUE_INJECT": "nan:17"})
    assert "B200 engine: dpd_engine_upload_beads failed" in log
    assert "stopped without save at time 2" in log
