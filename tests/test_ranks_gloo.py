"""The multi-process path of bench.py on the CPU: two ranks over gloo take
the run's collectives (a barrier, the maximum of the ranks' times), compute
the whole-job rate from the slowest rank, and step different replicas (each
rank its own seed); the reference arm runs on rank 0 only."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    try:
        import torch.distributed as dist
        import bench
        from osprey_dpd_b200 import ranks as R
        g = R.open_ranks("gloo", "cpu", timeout_s=60)
        local_ms = [10.0, 12.5][rank]
        g.barrier()
        mx = g.max(local_ms)
        value = R.aggregate_rate(g.world, 3000, 5, mx)
        system, _ = bench.workload("water", seed_offset=R.replica_seed_offset(rank))
        sums = [None] * world
        dist.all_gather_object(sums, float(np.sum(system.x)))
        g.barrier()
        g.close()
        q.put((rank, g.world, mx, value, sums))
    except Exception as exc:  # reported to the parent
        q.put((rank, "error", repr(exc)))


def test_two_gloo_ranks_time_and_replicas():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        item = q.get(timeout=180)
        res[item[0]] = item
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert res[r][1] != "error", res[r]
        _, world, mx, value, sums = res[r]
        assert world == 2
        assert mx == 12.5                              # the slowest rank's time, on every rank
        assert value == pytest.approx(2 * 3000 * 5 / 0.0125)
        assert sums[0] != sums[1]                      # independent replicas
    assert res[0][4] == res[1][4]


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    from osprey_dpd_b200 import ranks as R
    g = R.open_ranks("gloo", "cpu")
    assert (g.world, g.rank) == (1, 0)
    g.barrier()
    assert g.max(3.5) == 3.5
    g.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class Args:
        workload, steps, warmup = "bilayer", 3, 3

    assert bench.run_reference_arm(Args()) == 0
    assert capsys.readouterr().out == ""
