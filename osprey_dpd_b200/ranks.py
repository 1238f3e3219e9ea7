"""One process per GPU: the rank layout torchrun gives a run and the two
collectives a timed run takes -- a barrier on both sides of each timed
region and the maximum of the ranks' device times -- plus the whole-job
throughput computed from them.

In bench.py's multi-GPU runs every rank steps its own independent replica of
the workload (its own seed), so the only cross-rank traffic there is these
timing collectives; one box split over ranks is osprey_dpd_b200.slabs.  The
same code drives NCCL between GPUs and gloo between CPU processes (the
tests)."""
from __future__ import annotations

import datetime
import os
from typing import Optional


def layout() -> tuple:
    """(world size, rank, local rank) from torchrun's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed_offset(rank: int) -> int:
    """Seed offset of a rank's replica: every rank steps a different system."""
    return rank


def aggregate_rate(world: int, units_per_rank: int, steps: int, max_ms: float) -> float:
    """Whole-job units per second: all ranks' units over the slowest rank's time."""
    return world * units_per_rank * steps / (max_ms / 1000.0)


class Ranks:
    """The process group of a run (none for a single process).  `device` is
    where the reduction tensors live: the rank's GPU for NCCL, the CPU for
    gloo.  A short timeout makes ranks that wait for a missing peer end with
    an error instead of hanging."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 300.0):
        self.world, self.rank, self.local = layout()
        self.device = device
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    @property
    def dist(self):
        """The torch.distributed module when a process group is open, else None."""
        return self._dist

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """The maximum of x over the ranks (every rank gets it)."""
        if self._dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None


def open_ranks(backend: str = "nccl", device=None, timeout_s: float = 300.0) -> Optional[Ranks]:
    """Ranks for this process (a no-op group when WORLD_SIZE is 1)."""
    return Ranks(backend, device, timeout_s)
