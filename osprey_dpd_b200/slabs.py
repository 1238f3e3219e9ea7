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
form re-uploads each slab every step.

`SlabDecomposition.step_combined` is the same decomposition with ONE exchange
per step, the form the device slab engine runs: after a step each rank sends
a neighbour its migrants and, at once, the neighbour's ghosts for the next
step (its staying owned beads within `ghost` layers of that face), and keeps
its own migrants as ghosts (they lie in its ghost layer next to the face they
crossed).  `classify` is the per-bead rule of that exchange.

`DeviceSlabs` keeps each rank's slab resident on its GPU
(dpd_engine_slab_setup / _pack / _unpack of the C ABI): the classification,
the records, the next local box and its topology are formed by kernels; the
records travel between the ranks' device buffers over NCCL (or through host
copies over gloo)."""
from __future__ import annotations

import dataclasses
from typing import Callable, Dict, Optional

import numpy as np

# columns of a bead record (float64): id, type, movable, x(3), unPBC(3), v(3), f(3)
_COLS = 15

# output streams of an owned bead after a step (bits of `classify`)
TO_BELOW_MIG, TO_BELOW_GHOST, TO_ABOVE_MIG, TO_ABOVE_GHOST, KEEP = range(5)


def classify(lz: np.ndarray, owned: np.ndarray, g: int, own: int) -> np.ndarray:
    """Where each bead of a local box (local cell layer lz; layers g..g+own-1
    are the rank's own) goes after a step: an owned bead below layer g
    migrates to the rank below, one at or above g+own to the rank above;
    the others stay, and those within g layers of a face are also the next
    ghosts of the neighbour across it.  Ghosts go nowhere (their owners send
    them again).  Bits over (TO_BELOW_MIG, TO_BELOW_GHOST, TO_ABOVE_MIG,
    TO_ABOVE_GHOST, KEEP); the device form is slab_classify in
    osprey_dpd_b200/csrc/slab.cuh."""
    lz = np.asarray(lz)
    owned = np.asarray(owned, bool)
    m = np.zeros(len(lz), np.uint32)
    mb = owned & (lz < g)
    ma = owned & (lz >= g + own)
    stay = owned & ~mb & ~ma
    m[mb] |= 1 << TO_BELOW_MIG
    m[ma] |= 1 << TO_ABOVE_MIG
    m[stay] |= 1 << KEEP
    m[stay & (lz < 2 * g)] |= 1 << TO_BELOW_GHOST
    m[stay & (lz >= own)] |= 1 << TO_ABOVE_GHOST
    return m


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
        cols = to_below.shape[1]
        rb = torch.empty((int(n_from_below[1]), cols), dtype=torch.float64, device=dev)
        ra = torch.empty((int(n_from_above[0]), cols), dtype=torch.float64, device=dev)
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

    # ------------------------------------------------- one exchange per step
    def _combined_exchange(self, new: np.ndarray, lz: np.ndarray) -> None:
        """The owned beads `new` (global frame, after a step) in local layers
        lz: migrants and the neighbours' next ghosts out, the next owned
        beads and ghosts in (upload order of the device form: staying beads,
        migrants from below, from above; ghosts from below, from above, own
        migrants)."""
        m = classify(lz, np.ones(len(new), bool), self.ghost, self.z1 - self.z0)
        has = lambda k: (m >> k) & 1 == 1
        kind = lambda r, k: np.concatenate([r, np.full((len(r), 1), float(k))], axis=1)
        to_below = np.concatenate([kind(new[has(TO_BELOW_MIG)], 0), kind(new[has(TO_BELOW_GHOST)], 1)])
        to_above = np.concatenate([kind(new[has(TO_ABOVE_MIG)], 0), kind(new[has(TO_ABOVE_GHOST)], 1)])
        mine = np.concatenate([new[has(TO_BELOW_MIG)], new[has(TO_ABOVE_MIG)]])
        fb, fa = self._exchange(to_below, to_above)
        mig = lambda r: r[r[:, _COLS] == 0.0, :_COLS]
        gho = lambda r: r[r[:, _COLS] == 1.0, :_COLS]
        self.owned = np.concatenate([new[has(KEEP)], mig(fb), mig(fa)])
        self.ghosts = np.concatenate([gho(fb), gho(fa), mine])

    def start_combined(self) -> None:
        """The first exchange of the combined form (the first ghosts)."""
        self.ghosts = np.zeros((0, _COLS))
        if self.world > 1:
            lz = np.floor((self.owned[:, 5] + self._to_local(self.owned[:, 5])) / self.w).astype(np.int64)
            self._combined_exchange(self.owned, lz)

    def step_combined(self, t: int, make_engine: Callable, read_state: Callable) -> None:
        """One step of the local box (owned beads and the ghosts of the last
        exchange), then one exchange (start_combined first)."""
        own = self.owned
        rec = np.concatenate([own, self.ghosts])
        shift = self._to_local(rec[:, 5]) if self.world > 1 else np.zeros(len(rec))
        eng = make_engine(self._local_system(rec, shift))
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
        lz = np.floor(new[:, 5] / self.w).astype(np.int64)   # local frame
        new[:, 5] -= shift[:n_own]
        new[:, 8] -= self._u_shift()
        new[:, 5] = np.where(new[:, 5] < 0.0, new[:, 5] + self.Lz,
                             np.where(new[:, 5] >= self.Lz, new[:, 5] - self.Lz, new[:, 5]))
        self._combined_exchange(new, lz)

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


class DeviceSlabs:
    """One z-slab of `system`, resident on a GPU (dpd_engine_slab_*: the
    reference's mps* decomposition, mpsSimBox.cpp:796-860).  The local engine
    holds the slab's layers plus `ghost` layers on either side in the local
    frame (global z minus (z0 - ghost) * wz, wrapped); every step is
    dpd_engine_step followed by one exchange with the two neighbours (the
    combined form of SlabDecomposition.step_combined): the pack kernels write
    the records to send into device buffers, the buffers are swapped, and the
    unpack kernels form the next local box and its bonds on the device.

    With a process group (`group`, an osprey_dpd_b200.ranks.Ranks of two or
    more ranks, one slab per rank) the swap is NCCL point-to-point on the
    buffers themselves, or gloo through host copies when the group lives on
    the CPU.  Without one, `rank` and `world` name the slab and the slabs of
    a box are driven together in one process (`exchange_local`,
    `step_local`): the swap is then a device-to-device copy.  `device` is the
    CUDA ordinal; `capacity` the records one exchange buffer holds (default:
    room for 1.5 x the beads of ghost + 1 layers)."""

    def __init__(self, system, group=None, device: int = 0, ghost: int = 2, precision: int = None,
                 pair_scheme: int = None, capacity: int = None, rank: int = None, world: int = None):
        import torch
        from . import engine as E
        s = system
        self.sys, self.g = s, group
        self.world = group.world if group is not None else int(world)
        self.rank = group.rank if group is not None else int(rank)
        if self.world < 2:
            raise ValueError("a slab decomposition needs at least two slabs")
        nz = int(s.cells[2])
        self.w = float(s.widths[2])
        self.Lz = nz * self.w
        self.z0, self.z1 = slab_bounds(nz, self.world, self.rank)
        own = self.z1 - self.z0
        if ghost < 1 or own < 2 * ghost or own + 2 * ghost > nz:
            raise ValueError("every slab needs at least 2 * ghost cell layers, and slabs with their ghost "
                             "layers must be thinner than the box")
        self.ghost = ghost
        self.c = (self.z0 - ghost) * self.w
        self.dev = torch.device("cuda", device)
        self.eng = E.DpdEngine((s.cells[0], s.cells[1], own + 2 * ghost), s.widths, s.dt, s.lam, s.kT, s.a, s.gamma,
                               abs(int(s.seed)), E.MIXED if precision is None else precision, device)
        if pair_scheme is not None:
            self.eng.set_pair_scheme(pair_scheme)
        # one stream for the engine's kernels and the buffer traffic (torch's
        # default stream would leave the engine on its own, unordered with it)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.eng.set_stream(self.stream.cuda_stream)
        lay = np.floor(s.x[:, 2] / self.w).astype(np.int64)
        mine = np.nonzero((lay >= self.z0) & (lay < self.z1))[0]
        x = np.array(s.x[mine], np.float64)
        u = np.array(s.unpbc[mine], np.float64)
        x[:, 2] = np.mod(x[:, 2] - self.c, self.Lz)
        u[:, 2] -= self.c
        self.eng.upload_beads(s.ids[mine], s.types[mine], s.movable[mine], x, u, s.v[mine], s.f[mine])
        id_max = int(np.max(s.ids)) if len(s.ids) else 1
        self.eng.slab_setup(nz, self.z0, self.z1, ghost, len(mine), id_max, s.bond_head, s.bond_tail, s.bond_k2,
                            s.bond_l0, s.angle_first, s.angle_second, s.angle_k3, s.angle_phi0)
        self.n_owned, self.n_local = len(mine), len(mine)
        self.cap = int(capacity) if capacity else int(1.5 * (ghost + 1) * s.n / nz) + 256
        size = (self.cap + 1) * E.SLAB_RECORD
        # send below, send above, receive from below, receive from above
        with torch.cuda.stream(self.stream):
            self.bufs = [torch.zeros(size, dtype=torch.float64, device=self.dev) for _ in range(4)]
        if group is not None:
            self._exchange()

    # ------------------------------------------------------------ exchange
    def pack(self) -> None:
        sb, sa = self.bufs[0], self.bufs[1]
        self.eng.slab_pack(sb.data_ptr(), sa.data_ptr(), self.cap)

    def unpack(self) -> None:
        rb, ra = self.bufs[2], self.bufs[3]
        self.n_owned, self.n_local = self.eng.slab_unpack(rb.data_ptr(), ra.data_ptr())

    def _swap(self) -> None:
        """Send down and up, receive from above and below; posting order as in
        SlabDecomposition._exchange (with two ranks the one peer is both
        neighbours and messages match in posting order)."""
        import torch
        sb, sa, rb, ra = self.bufs
        dist = self.g.dist
        below, above = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        on_host = self.g.device is None or torch.device(self.g.device).type == "cpu"
        with torch.cuda.stream(self.stream):
            if on_host:
                hs = [sb.cpu(), sa.cpu()]
                hr = [torch.empty_like(hs[0]), torch.empty_like(hs[1])]
                ops = [dist.P2POp(dist.isend, hs[0], below), dist.P2POp(dist.isend, hs[1], above),
                       dist.P2POp(dist.irecv, hr[1], above), dist.P2POp(dist.irecv, hr[0], below)]
            else:
                ops = [dist.P2POp(dist.isend, sb, below), dist.P2POp(dist.isend, sa, above),
                       dist.P2POp(dist.irecv, ra, above), dist.P2POp(dist.irecv, rb, below)]
            for r in dist.batch_isend_irecv(ops):
                r.wait()
            if on_host:
                rb.copy_(hr[0])
                ra.copy_(hr[1])

    def _exchange(self) -> None:
        self.pack()
        self._swap()
        self.unpack()

    @staticmethod
    def exchange_local(slabs) -> None:
        """The exchange of all slabs of one box held by this process (one
        GPU): every slab packs, each receive buffer takes its neighbour's send
        buffer by a device copy, every slab unpacks."""
        import torch
        W = len(slabs)
        for sl in slabs:
            sl.pack()
        for sl in slabs:
            sl.stream.synchronize()           # every send buffer is written
        for r, sl in enumerate(slabs):
            below, above = slabs[(r - 1) % W], slabs[(r + 1) % W]
            with torch.cuda.stream(sl.stream):
                sl.bufs[2].copy_(below.bufs[1])   # the rank below sent it up
                sl.bufs[3].copy_(above.bufs[0])   # the rank above sent it down
        for sl in slabs:
            sl.stream.synchronize()           # no send buffer is read any more
        for sl in slabs:
            sl.unpack()

    @staticmethod
    def combine(parts, volume: float) -> Dict[str, float]:
        """The whole box's single-bead observables from the slabs' owned sums
        (dpd_engine_slab_observables): n, momentum, kT = sum v^2 / (3 n),
        the virial and P = (sum v^2 + trace virial) / (3 V) (CMonitor::
        CalculateSingleBeadData, Monitor.cpp:979-982)."""
        n = sum(p["n"] for p in parts)
        sv = np.sum([p["sum_v"] for p in parts], axis=0)
        sv2 = np.sum([p["sum_v2"] for p in parts], axis=0)
        vir = np.sum([p["virial"] for p in parts], axis=0)
        v2 = float(np.sum(sv2))
        has = all(p["has_virial"] for p in parts)
        return {"n": int(n), "sum_v": sv, "sum_v2": sv2, "virial": vir if has else None, "kT": v2 / (3.0 * n),
                "pressure": (v2 + vir[0] + vir[4] + vir[8]) / (3.0 * volume) if has else None}

    def volume(self) -> float:
        return float(np.prod(np.asarray(self.sys.cells, float) * np.asarray(self.sys.widths, float)))

    @staticmethod
    def step_local(slabs, t: int, observe: bool = False):
        """Step t of every slab held by this process, then the exchange; with
        observe, the whole box's observables of the step (combine)."""
        for sl in slabs:
            sl.eng.step(t, 1)
        obs = DeviceSlabs.combine([sl.eng.slab_observables() for sl in slabs], slabs[0].volume()) if observe \
            else None
        DeviceSlabs.exchange_local(slabs)
        return obs

    def step(self, t: int, observe: bool = False):
        """Step t of the local box, then the exchange (one slab per rank);
        with observe, the whole box's observables of the step (the owned sums
        all-reduced in FP64 over the process group)."""
        self.eng.step(t, 1)
        obs = self._observe() if observe else None
        self._exchange()
        return obs

    def _observe(self) -> Dict[str, float]:
        import torch
        p = self.eng.slab_observables()
        vec = np.concatenate([[p["n"]], p["sum_v"], p["sum_v2"], p["virial"], [1.0 if p["has_virial"] else 0.0]])
        dev = self.g.device if self.g.device is not None else "cpu"
        with torch.cuda.stream(self.stream):
            t = torch.tensor(vec, dtype=torch.float64, device=dev)
            self.g.dist.all_reduce(t)
            r = t.cpu().numpy()
        whole = {"n": int(round(r[0])), "sum_v": r[1:4], "sum_v2": r[4:7], "virial": r[7:16],
                 "has_virial": r[16] == self.world}
        return DeviceSlabs.combine([whole], self.volume())

    # -------------------------------------------------------------- state
    def owned_state(self) -> Dict[str, np.ndarray]:
        """This slab's owned beads (ids, global frame)."""
        d = self.eng.download(stress=False)
        ids, _ = self.eng.bead_ids()
        k = self.n_owned
        x, u = d["x"][:k].copy(), d["unpbc"][:k].copy()
        x[:, 2] += self.c
        x[:, 2] = np.where(x[:, 2] < 0.0, x[:, 2] + self.Lz, np.where(x[:, 2] >= self.Lz, x[:, 2] - self.Lz,
                                                                        x[:, 2]))
        u[:, 2] += self.c
        return {"id": ids[:k].copy(), "x": x, "unpbc": u, "v": d["v"][:k].copy(), "f": d["f"][:k].copy()}

    @staticmethod
    def merge(states) -> Dict[str, np.ndarray]:
        """owned_state of every slab -> the whole box by bead id."""
        out = {k: np.concatenate([a[k] for a in states]) for k in states[0]}
        order = np.argsort(out["id"])
        return {k: v[order] for k, v in out.items()}

    def gather(self) -> Optional[Dict[str, np.ndarray]]:
        """The whole box by bead id on rank 0 (None elsewhere; one slab per rank)."""
        mine = self.owned_state()
        allst = [None] * self.world
        self.g.dist.all_gather_object(allst, mine)
        return DeviceSlabs.merge(allst) if self.rank == 0 else None

    def close(self) -> None:
        self.eng.close()
