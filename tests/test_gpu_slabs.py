"""The z-slab decomposition (osprey_dpd_b200.slabs) with the GPU engine as
each rank's local engine: two gloo ranks (CPU processes sharing GPU 0; they
exchange ghosts and migrants on the host between steps, no kernel waits on
another rank) step a polymer solution whose bonds cross the slab faces; the
gathered box equals one FP64 engine stepping the whole box, to the rounding
that the atomic force sums leave."""
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 8


def _system():
    sys.path.insert(0, ROOT)
    from osprey_dpd_b200 import workloads as W
    return W.polymer_solution(cells=(6, 6, 12))


def _engine(s):
    from osprey_dpd_b200 import engine as E
    return E.DpdEngine.from_system(s, precision=E.FP64, device=0)


def _read(e):
    d = e.download(stress=False)
    e.close()
    return d


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    try:
        from osprey_dpd_b200 import ranks as R, slabs
        g = R.open_ranks("gloo", "cpu", timeout_s=300)
        dec = slabs.SlabDecomposition(_system(), g, ghost=2)
        for t in range(1, STEPS + 1):
            dec.step(t, _engine, _read)
        out = dec.gather()
        g.close()
        q.put((rank, out))
    except Exception:
        import traceback
        q.put((rank, "error", traceback.format_exc()))


def test_gpu_slabs_equal_single_box():
    s = _system()
    e = _engine(s)
    e.step(1, STEPS)
    ref = e.download(stress=False)
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
    got = res[0][1]
    order = np.argsort(s.ids)
    assert np.array_equal(got["id"], s.ids[order])
    for k, tol in (("x", 1e-8), ("unpbc", 1e-8), ("v", 1e-7), ("f", 1e-5)):
        np.testing.assert_allclose(got[k], ref[k][order], rtol=0, atol=tol)
