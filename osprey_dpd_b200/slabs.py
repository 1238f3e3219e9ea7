"""Spatial decomposition of one box into z-slabs, one per rank -- the
reference's own parallel design (its `mps*` boxes, SimBox.cpp:481-567) in
the simplest form that keeps every owned bead's step exact.

Each rank owns the beads in a contiguous range of CNT cell layers [z0, z1)
and, every step,

  1. sends the beads of its lowest and highest `ghost` layers to the ranks
     below and above (they are those ranks' ghost beads: position, unPBC
     position, velocity, last force, id, type);
  2. steps a local box of its own layers plus `ghost` layers on either side
     (periodic in z like the global box: with `ghost` >= 1 and at least
     2 * `ghost` owned layers the two ghost regions are never neighbours of
     an owned cell and no bead is both a lower and an upper boundary bead, so
     every pair, bond and angle with an owned bead is the reference's;
     results on ghosts are dropped);
  3. sends the owned beads that left its layers to the rank now owning them.

The pair noise is keyed on the two bead ids and the step (Philox), so an
owned bead feels exactly the random forces it feels in the single box and
no force is sent back.  One ghost layer covers the cut-off; the second covers
the drift of a step (beads move far less than a cell per step) and bonds
(partners within one cell).

The local engine is any object with the single-box step API: the GPU engine
(osprey_dpd_b200.engine.DpdEngine.from_system) or the CPU oracle.  This host
form re-uploads each slab every step; it fixes the data exchange the device
slab engine performs with kernels and NCCL."""
from __future__ import annotations

import dataclasses
from typing import Callable, Dict, Optional

import numpy as np

# columns of a bead record (float64): id, type, movable, x(3), unPBC(3), v(3), f(3)
_COLS = 15


def slab_bounds(nz: int, world: int, rank: int) -> tuple:
    """Cell layers [z0, z1) owned by `rank` (contiguous, sizes differ by at most one)."""
    base, extra = divmod(nz, world)
    z0 = rank * base + min(rank, extra)
    return z0, z0 + base + (1 if rank < extra else 0)


def _records(s, idx: np.ndarray) -> np.ndarray:
    r = np.empty((len(idx), _COLS))
    r[:, 0] = s.ids[idx]
    r[:, 1] = s.types[idx]
    r[:, 2] = s.movable[idx]
    r[:, 3:6] = s.x[idx]
    r[:, 6:9] = s.unpbc[idx]
    r[:, 9:12] = s.v[idx]
    r[:, 12:15] = s.f[idx]
    return r


class SlabDecomposition:
    """The owned beads of this rank and the per-step exchange.  `group` is an
    osprey_dpd_b200.ranks.Ranks (its process group carries the exchange);
    `system` is the global box (every rank holds the same copy at the start)."""

    def __init__(self, system, group, ghost: int = 2):
        self.sys = system
        self.g = group
        self.world, self.rank = group.world, group.rank
        nz = int(system.cells[2])
        self.w = float(system.widths[2])
        self.Lz = nz * self.w
        self.z0, self.z1 = slab_bounds(nz, self.world, self.rank)
        if ghost < 1:
            raise ValueError("ghost must be at least one cell layer")
        if self.world > 1:
            # a bead must not be both a lower and an upper boundary bead, and
            # no ghost may be an owned bead's own periodic image
            if self.z1 - self.z0 < 2 * ghost:
                raise ValueError("every rank needs at least 2 * ghost cell layers")
            if (self.z1 - self.z0) + 2 * ghost > nz:
                raise ValueError("slabs with their ghost layers must be thinner than the box")
        self.ghost = ghost if self.world > 1 else 0
        self.nzl = (self.z1 - self.z0) + 2 * self.ghost
        own = self._inside(system.x[:, 2], self.z0, self.z1)
        self.owned = _records(system, np.nonzero(own)[0])
        # global topology, by bead id (replicated)
        self.bond_head = np.asarray(system.bond_head, np.int64)
        self.bond_tail = np.asarray(system.bond_tail, np.int64)
        self.bond_k2 = np.asarray(system.bond_k2, np.float64)
        self.bond_l0 = np.asarray(system.bond_l0, np.float64)
        self.angle_first = np.asarray(system.angle_first, np.int64)
        self.angle_second = np.asarray(system.angle_second, np.int64)
        self.angle_k3 = np.asarray(system.angle_k3, np.float64)
        self.angle_phi0 = np.asarray(system.angle_phi0, np.float64)

    # --------------------------------------------------------------- geometry
    def _layer(self, z: np.ndarray) -> np.ndarray:
        return np.floor(z / self.w).astype(np.int64)

    def _inside(self, z: np.ndarray, z0: int, z1: int) -> np.ndarray:
        lay = self._layer(z)
        return (lay >= z0) & (lay < z1)

    def _to_local(self, z: np.ndarray) -> np.ndarray:
        """Shift that takes a global z of this slab or its ghosts into the
        local box [0, nzl w) (a ghost from across the global z face also
        takes the box's periodic shift)."""
        lz = np.mod(z - (self.z0 - self.ghost) * self.w, self.Lz)
        return lz - z

    def _u_shift(self) -> float:
        """The local frame's translation for unPBC positions: one constant for
        every bead, so bond vectors (unPBC differences) are unchanged."""
        return -(self.z0 - self.ghost) * self.w

    # --------------------------------------------------------------- exchange
    def _exchange(self, to_below: np.ndarray, to_above: np.ndarray):
        """(from_below, from_above): records sent by the neighbours.  Every
        rank posts its sends in the order (down, up) and its receives in the
        order (from above, from below): with two ranks the one peer is both
        neighbours, and messages between a pair match in posting order, so
        the peer's "down" records arrive as "from above" and its "up" records
        as "from below", as they must."""
        import torch
        dist = self.g.dist
        dev = self.g.device
        below, above = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        n_out = torch.tensor([len(to_below), len(to_above)], dtype=torch.int64, device=dev)
        n_from_below = torch.zeros(2, dtype=torch.int64, device=dev)
        n_from_above = torch.zeros(2, dtype=torch.int64, device=dev)
        ops = [dist.P2POp(dist.isend, n_out, below), dist.P2POp(dist.isend, n_out, above),
               dist.P2POp(dist.irecv, n_from_above, above), dist.P2POp(dist.irecv, n_from_below, below)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        # the rank below sent us its records for "above" (index 1), the rank above its "below" (index 0)
        rb = torch.empty((int(n_from_below[1]), _COLS), dtype=torch.float64, device=dev)
        ra = torch.empty((int(n_from_above[0]), _COLS), dtype=torch.float64, device=dev)
        sb = torch.as_tensor(np.ascontiguousarray(to_below)).to(dev)
        sa = torch.as_tensor(np.ascontiguousarray(to_above)).to(dev)
        ops = []
        if len(to_below):
            ops.append(dist.P2POp(dist.isend, sb, below))
        if len(to_above):
            ops.append(dist.P2POp(dist.isend, sa, above))
        if ra.shape[0]:
            ops.append(dist.P2POp(dist.irecv, ra, above))
        if rb.shape[0]:
            ops.append(dist.P2POp(dist.irecv, rb, below))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        return rb.cpu().numpy(), ra.cpu().numpy()

    # ------------------------------------------------------------------ step
    def _local_system(self, rec: np.ndarray, shift: np.ndarray):
        s = self.sys
        ids = rec[:, 0].astype(np.int64)
        x = rec[:, 3:6].copy()
        u = rec[:, 6:9].copy()
        x[:, 2] += shift
        u[:, 2] += self._u_shift()
        keep_b = np.isin(self.bond_head, ids) & np.isin(self.bond_tail, ids)
        bmap = -np.ones(len(keep_b), np.int64)
        bmap[keep_b] = np.arange(int(keep_b.sum()))
        keep_a = keep_b[self.angle_first] & keep_b[self.angle_second] if len(self.angle_first) else np.zeros(0, bool)
        local = dataclasses.replace(
            s, cells=(s.cells[0], s.cells[1], self.nzl), ids=ids, types=rec[:, 1].astype(np.int32),
            movable=rec[:, 2].astype(np.uint8), x=x, unpbc=u, v=rec[:, 9:12].copy(), f=rec[:, 12:15].copy(),
            bond_head=self.bond_head[keep_b], bond_tail=self.bond_tail[keep_b], bond_k2=self.bond_k2[keep_b],
            bond_l0=self.bond_l0[keep_b], angle_first=bmap[self.angle_first[keep_a]],
            angle_second=bmap[self.angle_second[keep_a]], angle_k3=self.angle_k3[keep_a],
            angle_phi0=self.angle_phi0[keep_a],
            bond_type=None if s.bond_type is None else np.asarray(s.bond_type)[keep_b],
            angle_type=None if s.angle_type is None else np.asarray(s.angle_type)[keep_a])
        return local

    def step(self, t: int, make_engine: Callable, read_state: Callable) -> None:
        """One step: ghosts in, the local box stepped by `make_engine(system)`
        (an engine holding that state; `read_state(engine)` returns its
        x, unpbc, v, f in the system's bead order), migrants out."""
        own = self.owned
        if self.world == 1:
            rec = own
            shift = np.zeros(len(own))
        else:
            lay = self._layer(own[:, 5])
            to_below = own[lay < self.z0 + self.ghost]
            to_above = own[lay >= self.z1 - self.ghost]
            from_below, from_above = self._exchange(to_below, to_above)
            rec = np.concatenate([own, from_below, from_above])
            shift = self._to_local(rec[:, 5])
        local = self._local_system(rec, shift)
        eng = make_engine(local)
        eng.step(t, 1)
        st = read_state(eng)
        n_own = len(own)
        new = own.copy()
        new[:, 3:6] = st["x"][:n_own]
        new[:, 6:9] = st["unpbc"][:n_own]
        new[:, 9:12] = st["v"][:n_own]
        new[:, 12:15] = st["f"][:n_own]
        if self.world == 1:
            self.owned = new
            return
        new[:, 5] -= shift[:n_own]
        new[:, 8] -= self._u_shift()
        # the global box's periodic wrap in z (the reference moves a bead by
        # one box length when it crosses a face)
        new[:, 5] = np.where(new[:, 5] < 0.0, new[:, 5] + self.Lz,
                             np.where(new[:, 5] >= self.Lz, new[:, 5] - self.Lz, new[:, 5]))
        lay = self._layer(new[:, 5])
        stay = (lay >= self.z0) & (lay < self.z1)
        nz = int(self.sys.cells[2])
        go_below = ~stay & (lay == (self.z0 - 1) % nz)
        go_above = ~stay & ~go_below
        in_below, in_above = self._exchange(new[go_below], new[go_above])
        self.owned = np.concatenate([new[stay], in_below, in_above])

    def gather(self) -> Optional[Dict[str, np.ndarray]]:
        """The whole box by bead id on rank 0 (None elsewhere)."""
        if self.world == 1:
            allrec = [self.owned]
        else:
            allrec = [None] * self.world
            self.g.dist.all_gather_object(allrec, self.owned)
        if self.rank != 0:
            return None
        rec = np.concatenate(allrec)
        rec = rec[np.argsort(rec[:, 0])]
        return {"id": rec[:, 0].astype(np.int64), "x": rec[:, 3:6], "unpbc": rec[:, 6:9], "v": rec[:, 9:12],
                "f": rec[:, 12:15]}
