"""Python binding of the C ABI in include/dpd_engine.h (ctypes).

This is a thin host-side mirror of the reference's per-step seam: create the
engine for a box (the CCNTCell statics), upload the beads and the bond/bond-pair
topology, step, and read back bead state and single-bead sums.  All work runs
in libospreydpd_cuda.so on the GPU; there is no CPU path, and loading fails
loudly when the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB

MIXED = 0
FP64 = 1

STATUS_CELL_SKIP = 0x1
STATUS_NONFINITE = 0x2
STATUS_IMAGE_OVERFLOW = 0x4
STATUS_INTERNAL = 0x8
STATUS_SLAB_REACH = 0x10

SLAB_RECORD = 16         # doubles per bead record of a slab exchange buffer

PAIR_FULL_SHELL = 0      # default: bitwise reproducible forces
PAIR_HALF_SHELL = 1      # each pair once, partner force by atomics
PAIR_STAGED = 2          # half shell with the neighbour rows staged in shared memory

EXPORTED = [
    "dpd_engine_create", "dpd_engine_upload_beads", "dpd_engine_upload_topology",
    "dpd_engine_set_pair_params", "dpd_engine_set_dt", "dpd_engine_set_thermostat",
    "dpd_engine_set_conservative", "dpd_engine_step", "dpd_engine_status", "dpd_engine_download",
    "dpd_engine_cells", "dpd_engine_observables", "dpd_engine_launch_count",
    "dpd_engine_last_error", "dpd_engine_destroy", "dpd_engine_set_stream", "dpd_engine_profile",
    "dpd_engine_profile_read", "dpd_engine_set_sample_period", "dpd_batch_create", "dpd_batch_upload_beads",
    "dpd_batch_observables", "dpd_engine_set_launch_shape", "dpd_engine_set_pair_scheme",
    "dpd_engine_set_slice_stress", "dpd_engine_slice_stress", "dpd_engine_set_monitor", "dpd_engine_monitor",
    "dpd_engine_set_restart_layout", "dpd_engine_write_restart", "dpd_engine_build_random",
    "dpd_write_paraview", "dpd_engine_write_paraview", "dpd_engine_renormalise_mom",
    "dpd_engine_slab_setup", "dpd_engine_slab_pack", "dpd_engine_slab_unpack", "dpd_engine_slab_counts",
    "dpd_engine_bead_ids", "dpd_engine_slab_observables", "dpd_engine_set_pair_tile", "dpd_engine_build_lamella",
]

KERNEL_NAMES = ["update_pos", "scan_cells", "permute", "gather", "pair_forces", "update_mom",
                "reduce_obs", "download", "kinetic", "bonds", "slices"]


class DpdParams(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("wx", C.c_double), ("wy", C.c_double), ("wz", C.c_double),
                ("dt", C.c_double), ("lam", C.c_double), ("kT", C.c_double),
                ("ntypes", C.c_int32), ("a", C.POINTER(C.c_double)), ("gamma", C.POINTER(C.c_double)),
                ("seed", C.c_uint64), ("precision", C.c_int32), ("device", C.c_int32)]


class DpdBox(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("wx", C.c_double), ("wy", C.c_double), ("wz", C.c_double),
                ("a", C.POINTER(C.c_double)), ("gamma", C.POINTER(C.c_double)), ("seed", C.c_uint64)]


class DpdMonitor(C.Structure):
    _fields_ = [("step", C.c_int64), ("n", C.c_int64), ("inertia", C.c_double * 9), ("bonds", C.c_int64),
                ("mean_bond_length", C.c_double), ("mean_sq_bond_length", C.c_double)]


class DpdObs(C.Structure):
    _fields_ = [("step", C.c_int64), ("n", C.c_int64), ("sum_v", C.c_double * 3), ("sum_v2", C.c_double * 3),
                ("virial", C.c_double * 9), ("sum_x", C.c_double * 3), ("ang_mom", C.c_double * 3),
                ("kT", C.c_double), ("pressure", C.c_double), ("has_virial", C.c_int32), ("pad", C.c_int32)]

    def as_dict(self) -> dict:
        return {"step": self.step, "n": self.n, "sum_v": list(self.sum_v), "sum_v2": list(self.sum_v2),
                "virial": list(self.virial), "sum_x": list(self.sum_x), "ang_mom": list(self.ang_mom),
                "kT": self.kT, "pressure": self.pressure, "has_virial": bool(self.has_virial)}


_lib = None


class EngineError(RuntimeError):
    pass


def load(path: Optional[str] = None) -> C.CDLL:
    """Loads libospreydpd_cuda.so; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise EngineError(f"{path} is missing: run `python -m osprey_dpd_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(path)
    vp = C.c_void_p
    L.dpd_engine_create.argtypes = [C.POINTER(DpdParams), C.POINTER(vp)]
    L.dpd_engine_upload_beads.argtypes = [vp, C.c_int64] + [vp] * 7
    L.dpd_engine_build_random.argtypes = [vp, C.c_int64, vp, vp, C.c_uint64, C.c_int64, C.c_int64, vp, vp, vp, vp]
    L.dpd_engine_build_lamella.argtypes = [vp, C.c_int64, vp, vp, C.c_int64, vp, vp, C.c_int32, C.c_int32, C.c_int32,
                                           C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_double, C.c_uint64,
                                           C.c_int64, C.c_int64, vp, vp, vp, vp]
    L.dpd_write_paraview.argtypes = [C.c_char_p, C.c_int64, vp, vp]
    L.dpd_engine_write_paraview.argtypes = [vp, C.c_char_p, vp, vp]
    L.dpd_engine_upload_topology.argtypes = [vp, C.c_int64, vp, vp, vp, vp, C.c_int64, vp, vp, vp, vp]
    L.dpd_engine_set_pair_params.argtypes = [vp, C.c_int32, vp, vp]
    L.dpd_engine_set_dt.argtypes = [vp, C.c_double]
    L.dpd_engine_set_thermostat.argtypes = [vp, C.c_int32]
    L.dpd_engine_set_conservative.argtypes = [vp, C.c_int32]
    L.dpd_engine_renormalise_mom.argtypes = [vp]
    L.dpd_engine_step.argtypes = [vp, C.c_int64, C.c_int32]
    L.dpd_engine_status.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.dpd_engine_download.argtypes = [vp] + [vp] * 5
    L.dpd_engine_cells.argtypes = [vp, vp]
    L.dpd_engine_observables.argtypes = [vp, C.POINTER(DpdObs)]
    L.dpd_engine_launch_count.argtypes = [vp]
    L.dpd_engine_launch_count.restype = C.c_int64
    L.dpd_engine_last_error.argtypes = [vp]
    L.dpd_engine_last_error.restype = C.c_char_p
    L.dpd_engine_set_stream.argtypes = [vp, vp]
    L.dpd_engine_set_sample_period.argtypes = [vp, C.c_int64]
    L.dpd_engine_set_launch_shape.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32]
    L.dpd_engine_set_pair_scheme.argtypes = [vp, C.c_int32]
    L.dpd_engine_set_pair_tile.argtypes = [vp, C.c_int32]
    L.dpd_engine_set_slice_stress.argtypes = [vp, C.c_int32, C.c_int32, vp, C.c_int32, vp]
    L.dpd_engine_set_monitor.argtypes = [vp, C.c_int32, vp, C.c_int32, vp, C.c_int64, vp, vp, vp, C.c_int32, vp]
    L.dpd_engine_monitor.argtypes = [vp, C.POINTER(DpdMonitor), vp, vp, vp, vp]
    L.dpd_engine_set_restart_layout.argtypes = [vp, C.c_int64, vp, vp, vp, vp]
    L.dpd_engine_write_restart.argtypes = [vp, C.c_char_p, C.c_int32, C.c_int32, C.c_int32]
    L.dpd_engine_slice_stress.argtypes = [vp, vp, vp, vp]
    L.dpd_engine_profile.argtypes = [vp, C.c_int32]
    L.dpd_engine_profile_read.argtypes = [vp, vp, vp]
    L.dpd_batch_create.argtypes = [C.POINTER(DpdParams), C.c_int32, C.POINTER(DpdBox), C.POINTER(vp)]
    L.dpd_batch_upload_beads.argtypes = [vp, C.c_int64] + [vp] * 8
    L.dpd_batch_observables.argtypes = [vp, C.c_int32, C.POINTER(DpdObs)]
    L.dpd_engine_slab_setup.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_int64,
                                        C.c_int64, vp, vp, vp, vp, C.c_int64, vp, vp, vp, vp]
    L.dpd_engine_slab_pack.argtypes = [vp, vp, vp, C.c_int64]
    L.dpd_engine_slab_unpack.argtypes = [vp, vp, vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.dpd_engine_slab_counts.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.dpd_engine_bead_ids.argtypes = [vp, vp, vp]
    L.dpd_engine_slab_observables.argtypes = [vp, C.POINTER(DpdObs)]
    L.dpd_engine_destroy.argtypes = [vp]
    L.dpd_engine_destroy.restype = None
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def write_paraview(path: str, x, display_id) -> None:
    """A Paraview snapshot of beads in file order from host arrays
    (dpd_write_paraview; needs no GPU)."""
    xv = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
    dv = np.ascontiguousarray(display_id, np.int32)
    if len(dv) != len(xv):
        raise ValueError("one display id per bead")
    rc = load().dpd_write_paraview(str(path).encode(), len(xv), _p(xv), _p(dv))
    if rc != 0:
        raise EngineError(f"dpd_write_paraview failed ({rc})")


def restart_layout(system):
    """(order, polymer id, polymer type) per bead of a workloads.DpdSystem in
    the reference's restart order: polymer by polymer, ids 1..N already in that
    order, polymer ids from 1."""
    pid, pty = [], []
    k = 1
    for t, p in enumerate(system.polymers):
        m = len(p.beads)
        pid.append(np.repeat(np.arange(k, k + p.count, dtype=np.int64), m))
        pty.append(np.full(p.count * m, t, dtype=np.int32))
        k += p.count
    order = np.arange(system.n, dtype=np.int64)
    return order, np.concatenate(pid), np.concatenate(pty)


def polymer_table(system):
    """(head id, tail id, polymer type) of every polymer of a workloads.DpdSystem:
    ids are 1..N in polymer order, each polymer's beads consecutive."""
    heads, tails, types = [], [], []
    nxt = 1
    for t, p in enumerate(system.polymers):
        m = len(p.beads)
        start = nxt + m * np.arange(p.count, dtype=np.int64)
        heads.append(start)
        tails.append(start + m - 1)
        types.append(np.full(p.count, t, dtype=np.int32))
        nxt += m * p.count
    cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt)
    return cat(heads, np.int64), cat(tails, np.int64), cat(types, np.int32)


class DpdEngine:
    """One engine instance: a box, its beads and topology, on one GPU."""

    def __init__(self, cells, widths, dt: float, lam: float, kT: float, a, gamma, seed: int,
                 precision: int = MIXED, device: int = -1):
        L = load()
        self._a = np.ascontiguousarray(a, dtype=np.float64)
        self._g = np.ascontiguousarray(gamma, dtype=np.float64)
        T = self._a.shape[0]
        p = DpdParams(int(cells[0]), int(cells[1]), int(cells[2]), float(widths[0]), float(widths[1]),
                      float(widths[2]), float(dt), float(lam), float(kT), T,
                      self._a.ctypes.data_as(C.POINTER(C.c_double)), self._g.ctypes.data_as(C.POINTER(C.c_double)),
                      int(seed) & 0xFFFFFFFFFFFFFFFF, int(precision), int(device))
        h = C.c_void_p()
        rc = L.dpd_engine_create(C.byref(p), C.byref(h))
        if rc != 0:
            raise EngineError(f"dpd_engine_create failed ({rc})")
        self.h = h
        self.n = 0
        self.precision = precision

    @classmethod
    def from_system(cls, system, precision: int = MIXED, device: int = -1, kT: float = None,
                    gamma_scale: float = 1.0, seed: int = None, topology: bool = True) -> "DpdEngine":
        eng = cls(system.cells, system.widths, system.dt, system.lam, system.kT if kT is None else kT,
                  system.a, system.gamma * gamma_scale, abs(int(system.seed if seed is None else seed)),
                  precision, device)
        eng.upload_beads(system.ids, system.types, system.movable, system.x, system.unpbc, system.v, system.f)
        if topology:
            eng.upload_topology(system.bond_head, system.bond_tail, system.bond_k2, system.bond_l0,
                                system.angle_first, system.angle_second, system.angle_k3, system.angle_phi0)
        return eng

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            msg = load().dpd_engine_last_error(self.h)
            raise EngineError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def upload_beads(self, ids, types, movable, x, unpbc, v, f=None) -> None:
        n = len(ids)
        arrs = [np.ascontiguousarray(ids, np.int64), np.ascontiguousarray(types, np.int32),
                None if movable is None else np.ascontiguousarray(movable, np.uint8),
                np.ascontiguousarray(x, np.float64), None if unpbc is None else np.ascontiguousarray(unpbc, np.float64),
                np.ascontiguousarray(v, np.float64), None if f is None else np.ascontiguousarray(f, np.float64)]
        self._check(load().dpd_engine_upload_beads(self.h, n, *[_p(a) for a in arrs]), "upload_beads")
        self.n = n

    def build_random(self, ids, types, seed: int, skip: int = 0, bond_head=None, bond_tail=None):
        """The random initial state of CRandomBuilder::Assemble built on the
        device and uploaded (dpd_engine_build_random); beads in the
        reference's creation order, bonds as bead indices in its polymer
        order.  Returns the built (x, v), each (n, 3), in that order."""
        n = len(ids)
        idv = np.ascontiguousarray(ids, np.int64)
        tv = np.ascontiguousarray(types, np.int32)
        bh = np.ascontiguousarray(bond_head if bond_head is not None else [], np.int64)
        bt = np.ascontiguousarray(bond_tail if bond_tail is not None else [], np.int64)
        x = np.zeros((n, 3))
        v = np.zeros((n, 3))
        self._check(load().dpd_engine_build_random(self.h, n, _p(idv), _p(tv), int(seed), int(skip), len(bh), _p(bh),
                                                   _p(bt), _p(x), _p(v)), "build_random")
        self.n = n
        return x, v

    def build_lamella(self, ids, types, poly_first, poly_type, lipid_type: int, head_offset: int, tail_offset: int,
                      normal: int = 2, centre: float = 0.5, thickness: float = 5.0, linearise: bool = True,
                      upper_fraction: float = 0.5, seed: int = 0, skip: int = 0, bond_head=None, bond_tail=None):
        """The lamella initial state of CLamellaBuilder::Assemble built on the
        device and uploaded (dpd_engine_build_lamella); beads in the
        reference's creation order, polymer p holding beads
        [poly_first[p], poly_first[p+1]).  Returns the built (x, v)."""
        n = len(ids)
        idv = np.ascontiguousarray(ids, np.int64)
        tv = np.ascontiguousarray(types, np.int32)
        pf = np.ascontiguousarray(poly_first, np.int64)
        pt = np.ascontiguousarray(poly_type, np.int32)
        bh = np.ascontiguousarray(bond_head if bond_head is not None else [], np.int64)
        bt = np.ascontiguousarray(bond_tail if bond_tail is not None else [], np.int64)
        x = np.zeros((n, 3))
        v = np.zeros((n, 3))
        self._check(load().dpd_engine_build_lamella(self.h, n, _p(idv), _p(tv), len(pt), _p(pf), _p(pt),
                                                    int(lipid_type), int(head_offset), int(tail_offset), int(normal),
                                                    float(centre), float(thickness), int(bool(linearise)),
                                                    float(upper_fraction), int(seed), int(skip), len(bh), _p(bh),
                                                    _p(bt), _p(x), _p(v)), "build_lamella")
        self.n = n
        return x, v

    def upload_topology(self, head, tail, k2, l0, first, second, k3, phi0) -> None:
        t = [np.ascontiguousarray(head, np.int64), np.ascontiguousarray(tail, np.int64),
             np.ascontiguousarray(k2, np.float64), np.ascontiguousarray(l0, np.float64),
             np.ascontiguousarray(first, np.int64), np.ascontiguousarray(second, np.int64),
             np.ascontiguousarray(k3, np.float64), np.ascontiguousarray(phi0, np.float64)]
        self._check(load().dpd_engine_upload_topology(self.h, len(t[0]), _p(t[0]), _p(t[1]), _p(t[2]), _p(t[3]),
                                                      len(t[4]), _p(t[4]), _p(t[5]), _p(t[6]), _p(t[7])),
                    "upload_topology")

    def slab_setup(self, nz_global: int, z0: int, z1: int, ghost: int, n_owned: int, id_max: int, head, tail, k2,
                   l0, first, second, k3, phi0) -> None:
        """dpd_engine_slab_setup: this engine becomes the slab [z0, z1) of a box
        of nz_global layers; the topology is the whole box's, by bead id."""
        t = [np.ascontiguousarray(head, np.int64), np.ascontiguousarray(tail, np.int64),
             np.ascontiguousarray(k2, np.float64), np.ascontiguousarray(l0, np.float64),
             np.ascontiguousarray(first, np.int64), np.ascontiguousarray(second, np.int64),
             np.ascontiguousarray(k3, np.float64), np.ascontiguousarray(phi0, np.float64)]
        self._check(load().dpd_engine_slab_setup(self.h, int(nz_global), int(z0), int(z1), int(ghost), int(n_owned),
                                                 int(id_max), len(t[0]), _p(t[0]), _p(t[1]), _p(t[2]), _p(t[3]),
                                                 len(t[4]), _p(t[4]), _p(t[5]), _p(t[6]), _p(t[7])), "slab_setup")

    def slab_pack(self, send_below: int, send_above: int, capacity: int) -> None:
        """dpd_engine_slab_pack into two device buffers (addresses) of
        (capacity + 1) * SLAB_RECORD doubles."""
        self._check(load().dpd_engine_slab_pack(self.h, C.c_void_p(int(send_below)), C.c_void_p(int(send_above)),
                                                int(capacity)), "slab_pack")

    def slab_unpack(self, recv_below: int, recv_above: int) -> tuple:
        """dpd_engine_slab_unpack from two device buffers; returns (owned, local) bead counts."""
        no, nl = C.c_int64(0), C.c_int64(0)
        self._check(load().dpd_engine_slab_unpack(self.h, C.c_void_p(int(recv_below)), C.c_void_p(int(recv_above)),
                                                  C.byref(no), C.byref(nl)), "slab_unpack")
        self.n = int(nl.value)
        return int(no.value), int(nl.value)

    def slab_observables(self) -> dict:
        """dpd_engine_slab_observables: the owned beads' single-bead sums
        (after a step, before the exchange)."""
        o = DpdObs()
        self._check(load().dpd_engine_slab_observables(self.h, C.byref(o)), "slab_observables")
        return o.as_dict()

    def slab_counts(self) -> tuple:
        no, nl = C.c_int64(0), C.c_int64(0)
        self._check(load().dpd_engine_slab_counts(self.h, C.byref(no), C.byref(nl)), "slab_counts")
        return int(no.value), int(nl.value)

    def set_pair_params(self, a, gamma) -> None:
        a = np.ascontiguousarray(a, np.float64)
        g = np.ascontiguousarray(gamma, np.float64)
        self._check(load().dpd_engine_set_pair_params(self.h, a.shape[0], _p(a), _p(g)), "set_pair_params")

    def set_dt(self, dt: float) -> None:
        self._check(load().dpd_engine_set_dt(self.h, float(dt)), "set_dt")

    def set_thermostat(self, on: bool) -> None:
        self._check(load().dpd_engine_set_thermostat(self.h, int(bool(on))), "set_thermostat")

    def set_conservative(self, on: bool) -> None:
        self._check(load().dpd_engine_set_conservative(self.h, int(bool(on))), "set_conservative")

    def renormalise_mom(self) -> None:
        self._check(load().dpd_engine_renormalise_mom(self.h), "renormalise_mom")

    def step(self, first_step: int, nsteps: int) -> None:
        self._check(load().dpd_engine_step(self.h, int(first_step), int(nsteps)), "step")

    def status(self) -> int:
        bits = C.c_uint32(0)
        self._check(load().dpd_engine_status(self.h, C.byref(bits)), "status")
        return int(bits.value)

    def download(self, stress: bool = True) -> dict:
        n = self.n
        out = {k: np.zeros((n, 3)) for k in ("x", "unpbc", "v", "f")}
        out["stress"] = np.zeros((n, 9)) if stress else None
        self._check(load().dpd_engine_download(self.h, _p(out["x"]), _p(out["unpbc"]), _p(out["v"]), _p(out["f"]),
                                               _p(out["stress"])), "download")
        return out

    def download_into(self, x=None, unpbc=None, v=None, f=None, stress=None) -> None:
        self._check(load().dpd_engine_download(self.h, _p(x), _p(unpbc), _p(v), _p(f), _p(stress)), "download")

    def bead_ids(self) -> tuple:
        """(ids, types) in upload order."""
        ids = np.zeros(self.n, np.int64)
        types = np.zeros(self.n, np.int32)
        self._check(load().dpd_engine_bead_ids(self.h, _p(ids), _p(types)), "bead_ids")
        return ids, types

    def cells(self) -> np.ndarray:
        c = np.zeros(self.n, dtype=np.int32)
        self._check(load().dpd_engine_cells(self.h, _p(c)), "cells")
        return c

    def observables(self) -> dict:
        o = DpdObs()
        self._check(load().dpd_engine_observables(self.h, C.byref(o)), "observables")
        return o.as_dict()

    def set_launch_shape(self, hitcap: int = 32, persistent_blocks_per_sm: int = 0, carveout: int = -1) -> None:
        self._check(load().dpd_engine_set_launch_shape(self.h, int(hitcap), int(persistent_blocks_per_sm),
                                                       int(carveout)), "set_launch_shape")

    def set_slice_stress(self, nslices: int, bond_type=None, nbondtypes: int = 0, bondpair_type=None,
                         nbptypes: int = 0) -> None:
        """Slice stress profile over ``nslices`` z slices on sample steps
        (CMonitor::AddBeadStress & co.); 0 turns it off."""
        self._sl_bt = np.ascontiguousarray(bond_type if bond_type is not None else [], np.int32)
        self._sl_bpt = np.ascontiguousarray(bondpair_type if bondpair_type is not None else [], np.int32)
        self._check(load().dpd_engine_set_slice_stress(self.h, int(nslices), int(nbondtypes), _p(self._sl_bt),
                                                       int(nbptypes), _p(self._sl_bpt)), "set_slice_stress")
        self._slice_dims = (int(nslices), int(self._a.shape[0]), int(nbondtypes), int(nbptypes))

    def set_monitor_for(self, system, initial_unpbc=None) -> None:
        """CMonitor sample data (dpd_engine_set_monitor) for a workloads.DpdSystem;
        initial unPBC positions in upload order, default the current ones."""
        ph, pt, pty = polymer_table(system)
        self._mon = dict(bt=np.ascontiguousarray(system.bond_type if system.bond_type is not None else [], np.int32),
                         at=np.ascontiguousarray(system.angle_type if system.angle_type is not None else [], np.int32),
                         ph=ph, pt=pt, pty=pty,
                         u0=None if initial_unpbc is None else np.ascontiguousarray(initial_unpbc, np.float64))
        m = self._mon
        self._mon_dims = (int(self._a.shape[0]), len(system.bond_specs), len(system.polymers),
                          len(system.bondpair_specs))
        self._check(load().dpd_engine_set_monitor(self.h, len(system.bond_specs), _p(m["bt"]),
                                                  len(system.bondpair_specs), _p(m["at"]), len(ph), _p(ph), _p(pt),
                                                  _p(pty), len(system.polymers), _p(m["u0"])), "set_monitor")

    def monitor(self) -> dict:
        """dpd_engine_monitor as a dict (see include/dpd_engine.h)."""
        T, nbt, npt, nbpt = getattr(self, "_mon_dims", (int(self._a.shape[0]), 0, 0, 0))
        o = DpdMonitor()
        msd, bl, ee, bp = np.zeros(T), np.zeros(nbt), np.zeros(npt), np.zeros((nbpt, 6))
        self._check(load().dpd_engine_monitor(self.h, C.byref(o), _p(msd), _p(bl), _p(ee), _p(bp)), "monitor")
        return {"step": o.step, "n": o.n, "inertia": np.array(o.inertia[:]).reshape(3, 3), "bonds": o.bonds,
                "mean_bond_length": o.mean_bond_length, "mean_sq_bond_length": o.mean_sq_bond_length,
                "msd": msd, "bond_length": bl, "end_to_end": ee, "bondpair": bp}

    def set_restart_layout_for(self, system, radius: float = 0.5) -> None:
        """dpd_engine_set_restart_layout for a workloads.DpdSystem (bead radius
        0.5 for every type, as the workloads' input files declare)."""
        order, pid, pty = restart_layout(system)
        self._rs = (order, pid, pty, np.full(self._a.shape[0], float(radius)))
        self._check(load().dpd_engine_set_restart_layout(self.h, len(order), *[_p(a) for a in self._rs]),
                    "set_restart_layout")

    def write_paraview(self, path: str, type_visible=None, display_id=None) -> None:
        """The current state as a Paraview snapshot (dpd_engine_write_paraview):
        beads by CNT cell, optional per-type visibility and per-bead display ids."""
        tv = None if type_visible is None else np.ascontiguousarray(type_visible, np.uint8)
        di = None if display_id is None else np.ascontiguousarray(display_id, np.int32)
        self._check(load().dpd_engine_write_paraview(self.h, str(path).encode(), _p(tv), _p(di)), "write_paraview")

    def write_restart(self, path: str, wall: bool = False, gravity: bool = False, shear: bool = False) -> None:
        self._check(load().dpd_engine_write_restart(self.h, os.fsencode(path), int(wall), int(gravity), int(shear)),
                    "write_restart")

    def set_slice_stress_for(self, system, nslices: int) -> None:
        """set_slice_stress with the bond and bond-pair types of a workloads.DpdSystem."""
        self.set_slice_stress(nslices, system.bond_type, len(system.bond_specs), system.angle_type,
                              len(system.bondpair_specs))

    def slice_stress(self) -> dict:
        """{"pair": [S][T*T][9], "bond": [S][NBT][9], "bondpair": [S][NBPT][9]}
        of the latest sample step."""
        dims = getattr(self, "_slice_dims", None)
        if dims is None or dims[0] == 0:   # off: let the engine report it
            self._check(load().dpd_engine_slice_stress(self.h, None, None, None), "slice_stress")
        S, T, nbt, nbpt = dims
        out = {"pair": np.zeros((S, T * T, 9)), "bond": np.zeros((S, nbt, 9)), "bondpair": np.zeros((S, nbpt, 9))}
        self._check(load().dpd_engine_slice_stress(self.h, _p(out["pair"]), _p(out["bond"]), _p(out["bondpair"])),
                    "slice_stress")
        return out

    def set_pair_scheme(self, scheme: int) -> None:
        """PAIR_FULL_SHELL (reproducible), PAIR_HALF_SHELL (each pair once) or
        PAIR_STAGED (each pair once, neighbour rows staged in shared memory)."""
        self._check(load().dpd_engine_set_pair_scheme(self.h, int(scheme)), "set_pair_scheme")

    def set_pair_tile(self, beads_per_block: int) -> None:
        """Beads per block of the half-shell kernel: 64 (default) or 128."""
        self._check(load().dpd_engine_set_pair_tile(self.h, int(beads_per_block)), "set_pair_tile")

    def set_sample_period(self, period: int) -> None:
        self._check(load().dpd_engine_set_sample_period(self.h, int(period)), "set_sample_period")

    def set_stream(self, stream_handle: int) -> None:
        """Queue on a caller's CUDA stream (e.g. torch.cuda.Stream().cuda_stream)."""
        self._check(load().dpd_engine_set_stream(self.h, C.c_void_p(int(stream_handle) or None)), "set_stream")

    def profile(self, on: bool) -> None:
        self._check(load().dpd_engine_profile(self.h, int(bool(on))), "profile")

    def profile_read(self) -> dict:
        ms = np.zeros(len(KERNEL_NAMES))
        cnt = np.zeros(len(KERNEL_NAMES), dtype=np.int64)
        self._check(load().dpd_engine_profile_read(self.h, _p(ms), _p(cnt)), "profile_read")
        return {k: {"ms": float(ms[i]), "launches": int(cnt[i])} for i, k in enumerate(KERNEL_NAMES)}

    def launch_count(self) -> int:
        return int(load().dpd_engine_launch_count(self.h))

    def close(self) -> None:
        h = getattr(self, "h", None)
        if h:
            load().dpd_engine_destroy(h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DpdBatch(DpdEngine):
    """Many independent boxes (replicas) advanced by the same kernel launches.

    ``systems`` are DpdSystem objects with the same bead types, dt, lambda and
    kT and no bonds; bead arrays in and out are the concatenation of the
    systems in order, positions box-local."""

    def __init__(self, systems, precision: int = MIXED, device: int = -1):
        L = load()
        s0 = systems[0]
        self.systems = list(systems)
        self._tabs = []
        boxes = (DpdBox * len(systems))()
        for k, s in enumerate(systems):
            a = np.ascontiguousarray(s.a, np.float64)
            g = np.ascontiguousarray(s.gamma, np.float64)
            self._tabs.append((a, g))
            boxes[k] = DpdBox(s.cells[0], s.cells[1], s.cells[2], *[float(w) for w in s.widths],
                              a.ctypes.data_as(C.POINTER(C.c_double)), g.ctypes.data_as(C.POINTER(C.c_double)),
                              abs(int(s.seed)) & 0xFFFFFFFFFFFFFFFF)
        self._a = self._tabs[0][0]
        self._g = self._tabs[0][1]
        p = DpdParams(0, 0, 0, 0.0, 0.0, 0.0, float(s0.dt), float(s0.lam), float(s0.kT), len(s0.type_names),
                      self._a.ctypes.data_as(C.POINTER(C.c_double)), self._g.ctypes.data_as(C.POINTER(C.c_double)),
                      0, int(precision), int(device))
        h = C.c_void_p()
        rc = L.dpd_batch_create(C.byref(p), len(systems), boxes, C.byref(h))
        if rc != 0:
            raise EngineError(f"dpd_batch_create failed ({rc})")
        self.h = h
        self.precision = precision
        self.offsets = np.cumsum([0] + [s.n for s in systems])
        cat = lambda f, dt: np.ascontiguousarray(np.concatenate([getattr(s, f) for s in systems]), dt)
        box = np.concatenate([np.full(s.n, k, np.int32) for k, s in enumerate(systems)])
        arrs = [box, cat("ids", np.int64), cat("types", np.int32), cat("movable", np.uint8), cat("x", np.float64),
                cat("unpbc", np.float64), cat("v", np.float64), cat("f", np.float64)]
        self.n = int(self.offsets[-1])
        self._check(L.dpd_batch_upload_beads(self.h, self.n, *[_p(a) for a in arrs]), "batch_upload_beads")

    def box_observables(self, box: int) -> dict:
        o = DpdObs()
        self._check(load().dpd_batch_observables(self.h, int(box), C.byref(o)), "batch_observables")
        return o.as_dict()

    def split(self, arr):
        return [arr[self.offsets[k]:self.offsets[k + 1]] for k in range(len(self.systems))]
