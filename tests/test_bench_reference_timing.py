"""The CPU reference timing of bench.py: the reference's step loop is run
twice from the same state (a third of the sample's steps, then all of them)
and the rate is the difference, so that what CSimBox::Run spends once before
its first step cancels.  A fake reference runner stands in for
oracle/_ref/osprey_ref_driver: only the arithmetic is under test."""
import importlib
import os
import sys

import pytest

from conftest import ROOT


@pytest.fixture
def bench_mod(monkeypatch):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dpd_oracle
    b = importlib.import_module("bench")
    calls = []

    def fake_run_reference(system, steps, dump=False, timeout=None):
        calls.append(steps)
        # 4 s spent once, then 0.5 s a step (or the table the test sets)
        t = fake_run_reference.table.get(steps, 4.0 + 0.5 * steps)
        return {"run_seconds": t, "bead_steps_per_s": system.n * steps / t}, None, None

    fake_run_reference.table = {}
    monkeypatch.setattr(dpd_oracle, "run_reference", fake_run_reference)
    monkeypatch.setattr(dpd_oracle, "REF_DRIVER", __file__)   # "built"
    return b, calls, fake_run_reference


class _Sys:
    n = 393216


def test_difference_cancels_the_one_time_cost(bench_mod):
    b, calls, _ = bench_mod
    cb = b.cpu_reference_sample(_Sys(), 12)
    assert calls == [4, 12]
    assert cb["steps"] == 8 and cb["kind"] == "reference" and cb["cores"] == 1
    assert cb["run_seconds"] == pytest.approx(4.0)
    assert cb["value"] == pytest.approx(_Sys.n / 0.5)   # the steady rate, not n * 12 / 10
    assert "differenced" in cb["sample"] and "12 minus 4 steps" in cb["sample"]


def test_one_step_sample_still_differences(bench_mod):
    b, calls, _ = bench_mod
    cb = b.cpu_reference_sample(_Sys(), 1)
    assert calls == [1, 2] and cb["steps"] == 1
    assert cb["value"] == pytest.approx(_Sys.n / 0.5)


def test_noise_larger_than_the_difference_falls_back_to_the_long_run(bench_mod):
    b, calls, fake = bench_mod
    fake.table = {4: 9.0, 12: 8.5}
    cb = b.cpu_reference_sample(_Sys(), 12)
    assert cb["steps"] == 12 and cb["run_seconds"] == pytest.approx(8.5)
    assert cb["value"] == pytest.approx(_Sys.n * 12 / 8.5)
