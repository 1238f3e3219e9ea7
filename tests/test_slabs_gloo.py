"""The z-slab decomposition (osprey_dpd_b200.slabs) on the CPU: two and three
gloo ranks, each stepping its slab plus ghost layers with the oracle (Philox
pair noise), exchange ghosts and migrants every step (in two exchanges, or in
the one combined exchange the device slab engine makes); the gathered box
equals the single-box oracle run to rounding (the summation order inside a
cell list differs).  A polymer solution (bonds across the slab faces and the
global z face) and a bilayer centred on a slab face (bonds and angles across
it)."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 10


def _system(kind="polymer"):
    sys.path.insert(0, ROOT)
    from osprey_dpd_b200 import workloads as W
    if kind == "bilayer":
        return W.bilayer(cells=(6, 6, 12), nlipids=40)
    return W.polymer_solution(cells=(6, 6, 12))


def _oracle_engine(s):
    import dpd_oracle as O
    return O.Oracle(s, noise=O.NOISE_PHILOX)


def _single_box(kind="polymer"):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    s = _system(kind)
    o = _oracle_engine(s)
    o.step(1, STEPS)
    st = o.state()
    order = np.argsort(s.ids)
    return {k: st[k][order] for k in ("x", "unpbc", "v", "f")}, s.ids[order]


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, q, kind="polymer", combined=False):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        from osprey_dpd_b200 import ranks as R, slabs
        g = R.open_ranks("gloo", "cpu", timeout_s=120)
        dec = slabs.SlabDecomposition(_system(kind), g, ghost=2)
        counts = []
        if combined:
            dec.start_combined()
        for t in range(1, STEPS + 1):
            if combined:
                dec.step_combined(t, _oracle_engine, lambda e: e.state())
            else:
                dec.step(t, _oracle_engine, lambda e: e.state())
            counts.append(len(dec.owned))
        out = dec.gather()
        g.close()
        q.put((rank, out, counts))
    except Exception as exc:
        import traceback
        q.put((rank, "error", traceback.format_exc()))


def _run(world, kind="polymer", combined=False):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, kind, combined)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        item = q.get(timeout=600)
        res[item[0]] = item
    for p in procs:
        p.join(timeout=60)
    for r in range(world):
        assert res[r][1] != "error", res[r][2]
    return res


def _compare(got, ref, ids):
    assert np.array_equal(got["id"], ids)
    np.testing.assert_allclose(got["x"], ref["x"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(got["unpbc"], ref["unpbc"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(got["v"], ref["v"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(got["f"], ref["f"], rtol=0, atol=1e-7)


@pytest.mark.parametrize("world,kind", [(2, "polymer"), (3, "polymer"), (2, "bilayer")])
def test_slabs_equal_single_box(world, kind):
    ref, ids = _single_box(kind)
    res = _run(world, kind)
    _compare(res[0][1], ref, ids)
    assert sum(res[r][2][-1] for r in range(world)) == len(ids)   # every bead owned once


@pytest.mark.parametrize("world,kind", [(2, "polymer"), (3, "polymer"), (2, "bilayer")])
def test_combined_exchange_equals_single_box(world, kind):
    """One exchange per step (migrants and the next ghosts together, the
    device slab engine's form) gives the same box."""
    ref, ids = _single_box(kind)
    res = _run(world, kind, combined=True)
    _compare(res[0][1], ref, ids)
    assert sum(res[r][2][-1] for r in range(world)) == len(ids)


def test_classify_rule():
    sys.path.insert(0, ROOT)
    from osprey_dpd_b200 import slabs as S
    g, own = 2, 5                       # local layers 0..8: ghosts 0,1 and 7,8
    lz = np.arange(-0, 9)
    m = S.classify(lz, np.ones(9, bool), g, own)
    bit = lambda k: [int(v) for v in (m >> k) & 1]
    assert bit(S.TO_BELOW_MIG) == [1, 1, 0, 0, 0, 0, 0, 0, 0]
    assert bit(S.TO_ABOVE_MIG) == [0, 0, 0, 0, 0, 0, 0, 1, 1]
    assert bit(S.KEEP) == [0, 0, 1, 1, 1, 1, 1, 0, 0]
    assert bit(S.TO_BELOW_GHOST) == [0, 0, 1, 1, 0, 0, 0, 0, 0]
    assert bit(S.TO_ABOVE_GHOST) == [0, 0, 0, 0, 0, 1, 1, 0, 0]
    assert not S.classify(lz, np.zeros(9, bool), g, own).any()   # ghosts go nowhere


def test_single_rank_is_the_box(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from osprey_dpd_b200 import ranks as R, slabs
    ref, ids = _single_box()
    dec = slabs.SlabDecomposition(_system(), R.open_ranks("gloo", "cpu"), ghost=2)
    for t in range(1, STEPS + 1):
        dec.step(t, _oracle_engine, lambda e: e.state())
    _compare(dec.gather(), ref, ids)


def test_slab_bounds_and_limits():
    sys.path.insert(0, ROOT)
    from osprey_dpd_b200 import slabs
    assert [slabs.slab_bounds(10, 3, r) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert slabs.slab_bounds(12, 1, 0) == (0, 12)


def test_combine_owned_sums():
    """DeviceSlabs.combine: kT = sum v^2 / 3N and P = (sum v^2 + trace W) / 3V
    of the whole box from the slabs' owned sums (CMonitor::
    CalculateSingleBeadData, Monitor.cpp:979-982)."""
    sys.path.insert(0, ROOT)
    from osprey_dpd_b200 import slabs as S
    parts = [{"n": 10, "sum_v": np.array([1.0, 0.0, -1.0]), "sum_v2": np.array([10.0, 11.0, 9.0]),
              "virial": np.arange(9.0), "has_virial": True},
             {"n": 20, "sum_v": np.array([-1.0, 0.5, 1.0]), "sum_v2": np.array([20.0, 19.0, 21.0]),
              "virial": np.ones(9), "has_virial": True}]
    o = S.DeviceSlabs.combine(parts, volume=100.0)
    assert o["n"] == 30
    np.testing.assert_allclose(o["sum_v"], [0.0, 0.5, 0.0])
    assert o["kT"] == (30.0 + 60.0) / 90.0
    tr = (0.0 + 4.0 + 8.0) + 3.0
    assert o["pressure"] == (90.0 + tr) / 300.0
    parts[1]["has_virial"] = False
    assert S.DeviceSlabs.combine(parts, 100.0)["pressure"] is None
