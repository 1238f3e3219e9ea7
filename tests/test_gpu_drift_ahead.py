"""The drift done ahead: the last k_update_mom of a call also performs the
next call's UpdatePos into separate buffers, so a following call starts at
its cell sort.  It must not change any result: with the bitwise
reproducible full-shell scheme in FP64, a run of single-step calls equals
the same run with the drift-ahead turned off (DPD_TUNE=ahead=0) bit for bit,
also across downloads, a time-step change and a re-upload, and equals one
multi-step call."""
import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _engine(engine_mod, s, monkeypatch, ahead):
    monkeypatch.setenv("DPD_TUNE", "ahead=1" if ahead else "ahead=0")
    e = engine_mod.DpdEngine.from_system(s, precision=1)
    monkeypatch.delenv("DPD_TUNE")
    return e


def _same(a, b):
    ga, gb = a.download(), b.download()
    for k in ("x", "unpbc", "v", "f"):
        assert np.array_equal(ga[k], gb[k]), k
    assert np.array_equal(a.cells(), b.cells())


def test_single_step_calls_equal_without_drift_ahead(engine_mod, monkeypatch):
    s = W.bilayer(cells=(10, 10, 10), nlipids=30)
    on = _engine(engine_mod, s, monkeypatch, True)
    off = _engine(engine_mod, s, monkeypatch, False)
    for t in range(1, 9):
        on.step(t, 1)
        off.step(t, 1)
        if t % 3 == 0:
            _same(on, off)   # downloads between calls see the step's own state
    _same(on, off)
    assert on.observables()["sum_v2"] == off.observables()["sum_v2"]
    assert on.status() == 0 and off.status() == 0


def test_call_lengths_time_step_change_and_reupload(engine_mod, monkeypatch):
    s = W.binary_mixture(cells=(8, 9, 10))
    on = _engine(engine_mod, s, monkeypatch, True)
    off = _engine(engine_mod, s, monkeypatch, False)
    t = 1
    for k in (1, 3, 1, 2):
        on.step(t, k)
        off.step(t, k)
        t += k
    _same(on, off)
    # a time-step change between calls: the drift done ahead used the old dt
    on.set_dt(0.01)
    off.set_dt(0.01)
    on.step(t, 1)
    off.step(t, 1)
    t += 1
    _same(on, off)
    on.step(t, 2)
    off.step(t, 2)
    t += 2
    _same(on, off)
    # a re-upload replaces the drifted state: afterwards the engine steps as a
    # fresh one created from the new state (same seed, so the same noise)
    s2 = W.binary_mixture(cells=(8, 9, 10), seed=77)
    on.upload_beads(s2.ids, s2.types, s2.movable, s2.x, s2.unpbc, s2.v, s2.f)
    monkeypatch.setenv("DPD_TUNE", "ahead=0")
    fresh = engine_mod.DpdEngine.from_system(s2, precision=1, seed=s.seed)
    monkeypatch.delenv("DPD_TUNE")
    fresh.set_dt(0.01)
    on.step(1, 1)
    fresh.step(1, 1)
    on.step(2, 2)
    fresh.step(2, 2)
    _same(on, fresh)


def test_single_step_calls_equal_one_long_call(engine_mod, monkeypatch):
    s = W.polymer_solution(cells=(9, 9, 9))
    a = _engine(engine_mod, s, monkeypatch, True)
    b = _engine(engine_mod, s, monkeypatch, True)
    # no sample step in either run: the sampling kernel variants may round differently
    a.set_sample_period(1000)
    b.set_sample_period(1000)
    for t in range(1, 7):
        a.step(t, 1)
    b.step(1, 6)
    _same(a, b)
