"""Replica batches: many A/B boxes of different size, a_AB and seed advanced
by the same kernel launches must evolve exactly as each box does in its own
engine (same kernels, same per-box cell order, same noise stream)."""
import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _replicas(k=7, lo=3, hi=9):
    edges, fracs, a_ab, seeds = W.replica_table(k, lo=lo, hi=hi)
    return [W.binary_mixture(n=int(edges[r]), seed=int(seeds[r]), a_ab=float(a_ab[r]), frac_a=float(fracs[r]))
            for r in range(k)]


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_batch_equals_replicas_run_alone(engine_mod, precision):
    systems = _replicas()
    batch = engine_mod.DpdBatch(systems, precision=precision)
    batch.step(1, 12)
    got = batch.download()
    cells = batch.cells()
    assert batch.status() & ~engine_mod.STATUS_CELL_SKIP == 0
    for k, s in enumerate(systems):
        eng = engine_mod.DpdEngine.from_system(s, precision=precision, topology=False)
        eng.step(1, 12)
        ref = eng.download()
        for key in ("x", "unpbc", "v", "f", "stress"):
            assert np.array_equal(batch.split(got[key])[k], ref[key]), (k, key)
        assert np.array_equal(batch.split(cells)[k], eng.cells())
        ob, oe = batch.box_observables(k), eng.observables()
        assert ob["n"] == s.n
        assert np.allclose(ob["sum_v2"], oe["sum_v2"], rtol=1e-12, atol=0)
        assert np.allclose(ob["virial"], oe["virial"], rtol=1e-9, atol=1e-9)
        eng.close()


def test_batch_matches_oracle_per_box(engine_mod, oracle_mod):
    from conftest import rel_err
    systems = _replicas(4, 4, 7)
    batch = engine_mod.DpdBatch(systems, precision=1)
    batch.step(1, 3)
    f = batch.split(batch.download()["f"])
    for k, s in enumerate(systems):
        o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
        o.step(1, 3)
        assert rel_err(f[k], o.state()["f"]) < 1e-10
