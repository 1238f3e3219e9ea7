"""The device-resident z-slab decomposition (dpd_engine_slab_*, driven by
osprey_dpd_b200.slabs.DeviceSlabs) against one engine stepping the whole box.

* In one process: the slabs of a box on GPU 0, their exchange buffers swapped
  by device copies (no collectives, no kernel waits on another); two and three
  slabs of a polymer solution (bonds across the slab faces and the global z
  face), of a bilayer centred on a slab face (bonds and bond pairs across
  it) and of an A/B mixture, FP64; a mixed-precision run; every bead owned by
  exactly one slab.
* Two gloo ranks (CPU processes sharing GPU 0) with DeviceSlabs over the
  process group (buffers swapped through host copies).
* The checks: a bond reaching beyond the ghost layers (fatal status), an
  exchange buffer too small (DPD_E_LIMIT on every slab), bad geometry.

Bounds against the single box, FP64: the pair forces of a slab are summed
over another cell order, and 8 steps amplify that rounding (x, unPBC 1e-8;
v 1e-7; F 1e-5, the bounds of the host-form slab test)."""
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 8


def _system(kind="polymer"):
    sys.path.insert(0, ROOT)
    from osprey_dpd_b200 import workloads as W
    if kind == "bilayer":
        return W.bilayer(cells=(6, 6, 12), nlipids=40)
    if kind == "binary":
        return W.binary_mixture(cells=(6, 6, 12))
    if kind == "water":
        return W.water(6)
    return W.polymer_solution(cells=(6, 6, 12))


def _single_box(s, precision, steps=STEPS):
    from osprey_dpd_b200 import engine as E
    e = E.DpdEngine.from_system(s, precision=precision, device=0)
    e.step(1, steps)
    d = e.download(stress=False)
    e.close()
    order = np.argsort(s.ids)
    return {k: d[k][order] for k in ("x", "unpbc", "v", "f")}, s.ids[order]


def _compare(got, ref, ids, tol=(1e-8, 1e-8, 1e-7, 1e-5)):
    assert np.array_equal(got["id"], ids)
    for k, t in zip(("x", "unpbc", "v", "f"), tol):
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=t, err_msg=k)


def _local_run(s, world, precision, steps=STEPS, **kw):
    from osprey_dpd_b200 import slabs as S
    slabs = [S.DeviceSlabs(s, None, device=0, rank=r, world=world, precision=precision, **kw) for r in range(world)]
    S.DeviceSlabs.exchange_local(slabs)          # the first ghosts
    owned = []
    for t in range(1, steps + 1):
        S.DeviceSlabs.step_local(slabs, t)
        owned.append(sum(sl.n_owned for sl in slabs))
    got = S.DeviceSlabs.merge([sl.owned_state() for sl in slabs])
    status = [sl.eng.status() for sl in slabs]
    for sl in slabs:
        sl.close()
    return got, owned, status


@pytest.mark.parametrize("world,kind", [(2, "polymer"), (3, "polymer"), (2, "bilayer"), (3, "binary")])
def test_device_slabs_equal_single_box(world, kind):
    from osprey_dpd_b200 import engine as E
    s = _system(kind)
    ref, ids = _single_box(s, E.FP64)
    got, owned, status = _local_run(s, world, E.FP64)
    assert owned == [s.n] * STEPS                  # every bead owned by exactly one slab
    assert all(st == 0 for st in status)
    _compare(got, ref, ids)


def test_device_slab_observables():
    """The slabs' owned-bead sums combined (kT, pressure, virial; full-shell
    FP64, every step a sample step) equal the whole box's observables."""
    from osprey_dpd_b200 import engine as E, slabs as S
    s = _system("bilayer")
    e = E.DpdEngine.from_system(s, precision=E.FP64, device=0)
    e.step(1, 4)
    ref = e.observables()
    e.close()
    slabs = [S.DeviceSlabs(s, None, device=0, rank=r, world=2, precision=E.FP64) for r in range(2)]
    S.DeviceSlabs.exchange_local(slabs)
    for t in range(1, 5):
        obs = S.DeviceSlabs.step_local(slabs, t, observe=True)
    for sl in slabs:
        sl.close()
    assert obs["n"] == s.n
    assert abs(obs["kT"] - ref["kT"]) <= 1e-10 * ref["kT"]
    assert abs(obs["pressure"] - ref["pressure"]) <= 1e-9 * abs(ref["pressure"])
    scale = float(np.max(np.abs(ref["virial"])))
    np.testing.assert_allclose(obs["virial"], ref["virial"], rtol=0, atol=1e-9 * scale)
    np.testing.assert_allclose(obs["sum_v"], ref["sum_v"], rtol=0, atol=1e-9)


def test_device_slabs_mixed_precision():
    """Mixed precision, half-shell pair scheme: 3 steps within the
    mixed-precision bounds of the parity tests (1e-4 of the RMS)."""
    from osprey_dpd_b200 import engine as E
    s = _system("polymer")
    e = E.DpdEngine.from_system(s, precision=E.MIXED, device=0)
    e.set_pair_scheme(E.PAIR_HALF_SHELL)
    e.step(1, 3)
    d = e.download(stress=False)
    e.close()
    order = np.argsort(s.ids)
    got, owned, status = _local_run(s, 2, E.MIXED, steps=3, pair_scheme=E.PAIR_HALF_SHELL)
    assert owned == [s.n] * 3 and status == [0, 0]
    for k in ("x", "v", "f"):
        r = d[k][order]
        scale = float(np.sqrt(np.mean(r * r)))
        assert np.max(np.abs(got[k] - r)) <= 1e-4 * scale, k


def test_bond_beyond_ghost_layers_is_fatal():
    """A bond from an owned bead to a bead outside the local box: after an
    exchange (here with empty neighbours) the slab's topology filter sets
    DPD_STATUS_SLAB_REACH and the next step refuses."""
    import torch
    from osprey_dpd_b200 import engine as E
    s = _system("water")
    w = float(s.widths[2])
    nz = int(s.cells[2])
    lay = np.floor(s.x[:, 2] / w).astype(int)
    z0, z1, g = 0, nz // 2, 1
    mine = np.nonzero((lay >= z0) & (lay < z1))[0]
    far = np.nonzero(lay == nz - 2)[0][0]          # two layers below the local box, periodically
    c = (z0 - g) * w
    eng = E.DpdEngine((s.cells[0], s.cells[1], z1 - z0 + 2 * g), s.widths, s.dt, s.lam, s.kT, s.a, s.gamma,
                      abs(int(s.seed)), E.FP64, 0)
    x = s.x[mine].copy()
    x[:, 2] = np.mod(x[:, 2] - c, nz * w)
    u = s.unpbc[mine].copy()
    u[:, 2] -= c
    eng.upload_beads(s.ids[mine], s.types[mine], None, x, u, s.v[mine], s.f[mine])
    head = int(s.ids[mine[0]])
    eng.slab_setup(nz, z0, z1, g, len(mine), int(s.ids.max()), [head], [int(s.ids[far])], [128.0], [0.5],
                   [], [], [], [])
    assert eng.status() == 0                       # no ghosts before the first exchange: no check
    cap = 512
    bufs = [torch.zeros((cap + 1) * E.SLAB_RECORD, dtype=torch.float64, device="cuda:0") for _ in range(4)]
    torch.cuda.synchronize()                       # the buffers are zeroed
    eng.slab_pack(bufs[0].data_ptr(), bufs[1].data_ptr(), cap)
    torch.cuda.synchronize()
    eng.slab_unpack(bufs[2].data_ptr(), bufs[3].data_ptr())   # nothing received
    assert eng.status() & E.STATUS_SLAB_REACH
    with pytest.raises(E.EngineError):
        eng.step(1, 1)
    eng.close()


def test_exchange_overflow_and_errors():
    from osprey_dpd_b200 import engine as E, slabs as S
    s = _system("polymer")
    slabs = [S.DeviceSlabs(s, None, device=0, rank=r, world=2, precision=E.FP64, capacity=8) for r in range(2)]
    import torch
    for sl in slabs:
        sl.pack()
    torch.cuda.synchronize()
    for r, sl in enumerate(slabs):
        sl.bufs[2].copy_(slabs[1 - r].bufs[1])
        sl.bufs[3].copy_(slabs[1 - r].bufs[0])
    torch.cuda.synchronize()
    for sl in slabs:
        with pytest.raises(E.EngineError, match="exchange buffers"):
            sl.unpack()
        with pytest.raises(E.EngineError):          # no pack pending
            sl.unpack()
        sl.close()
    with pytest.raises(ValueError):
        S.DeviceSlabs(s, None, device=0, rank=0, world=4)      # 3 layers per slab < 2 * ghost
    e = E.DpdEngine.from_system(s, precision=E.FP64, device=0, topology=False)
    with pytest.raises(E.EngineError):
        e.slab_pack(1 << 20, 2 << 20, 8)                        # not a slab
    with pytest.raises(E.EngineError):
        e.slab_setup(12, 0, 6, 2, e.n, 1, [], [], [], [], [], [], [], [])   # box holds 12 layers, not 10
    e.close()


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    try:
        from osprey_dpd_b200 import engine as E, ranks as R, slabs
        g = R.open_ranks("gloo", "cpu", timeout_s=300)
        dec = slabs.DeviceSlabs(_system(), g, device=0, precision=E.FP64)
        for t in range(1, STEPS + 1):
            obs = dec.step(t, observe=(t == STEPS))
        out = dec.gather()
        dec.close()
        g.close()
        q.put((rank, out, obs))
    except Exception:
        import traceback
        q.put((rank, "error", traceback.format_exc()))


def test_device_slabs_over_gloo_ranks():
    """Two ranks, buffers through host copies; the observables of the last
    step all-reduced over the group equal the whole box's."""
    from osprey_dpd_b200 import engine as E
    s = _system()
    ref, ids = _single_box(s, E.FP64)
    e = E.DpdEngine.from_system(s, precision=E.FP64, device=0)
    e.step(1, STEPS)
    ref_obs = e.observables()
    e.close()
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        item = q.get(timeout=600)
        res[item[0]] = item
    for p in procs:
        p.join(timeout=60)
    for r in range(2):
        assert res[r][1] != "error", res[r][2]
    _compare(res[0][1], ref, ids)
    for r in range(2):
        obs = res[r][2]
        assert obs["n"] == s.n
        assert abs(obs["kT"] - ref_obs["kT"]) <= 1e-9 * ref_obs["kT"]
        assert abs(obs["pressure"] - ref_obs["pressure"]) <= 1e-8 * abs(ref_obs["pressure"])


def test_slab_refuses_whole_box_calls():
    """A slab's local box also holds ghosts: the whole-box calls refuse it
    and name the slab form where there is one."""
    from osprey_dpd_b200 import engine as E, slabs as S
    s = _system("polymer")
    sl = S.DeviceSlabs(s, None, device=0, rank=0, world=2, precision=E.FP64)
    e = sl.eng
    for call in (lambda: e.observables(), lambda: e.renormalise_mom(), lambda: e.set_slice_stress_for(s, 4),
                 lambda: e.set_monitor_for(s), lambda: e.set_restart_layout_for(s),
                 lambda: e.upload_beads(s.ids, s.types, None, s.x, s.unpbc, s.v),
                 lambda: e.build_random(s.ids, s.types, 5),
                 lambda: e.upload_topology(s.bond_head, s.bond_tail, s.bond_k2, s.bond_l0, s.angle_first,
                                           s.angle_second, s.angle_k3, s.angle_phi0)):
        with pytest.raises(E.EngineError):
            call()
    sl.close()


def test_device_slabs_at_benchmark_size():
    """The benchmark's 393,216-bead H3T6 bilayer in four slabs (one process,
    FP64, full shell) against one engine stepping the whole box: 3 steps,
    every bead owned once, the same bounds as the small boxes."""
    from osprey_dpd_b200 import engine as E, workloads as W2
    s = W2.bilayer()
    ref, ids = _single_box(s, E.FP64, steps=3)
    got, owned, status = _local_run(s, 4, E.FP64, steps=3)
    assert owned == [s.n] * 3 and all(st == 0 for st in status)
    _compare(got, ref, ids)
