"""ctypes binding of the CPU oracle (dpd_oracle.c) and a runner for the
reference harness (ref_driver.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, never by the engine.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libdpd_oracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "osprey_ref_driver")

NOISE_LCG = 0
NOISE_PHILOX = 1


class _Params(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("wx", C.c_double), ("wy", C.c_double), ("wz", C.c_double),
                ("dt", C.c_double), ("lam", C.c_double), ("kT", C.c_double),
                ("ntypes", C.c_int32), ("a", C.POINTER(C.c_double)), ("gamma", C.POINTER(C.c_double)),
                ("seed", C.c_uint64), ("noise", C.c_int32)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.dpdo_create.restype = vp
        L.dpdo_create.argtypes = [C.POINTER(_Params)]
        L.dpdo_destroy.argtypes = [vp]
        L.dpdo_set_beads.argtypes = [vp, C.c_int64] + [vp] * 7
        L.dpdo_set_topology.argtypes = [vp, C.c_int64, vp, vp, vp, vp, C.c_int64, vp, vp, vp, vp]
        L.dpdo_step.argtypes = [vp, C.c_int64, C.c_int32]
        L.dpdo_get.argtypes = [vp] + [vp] * 5
        L.dpdo_get_cells.argtypes = [vp, vp]
        L.dpdo_cell_errors.argtypes = [vp]
        L.dpdo_cell_errors.restype = C.c_int64
        L.dpdo_pair_count.argtypes = [vp]
        L.dpdo_pair_count.restype = C.c_int64
        L.dpdo_philox_pair.argtypes = [C.c_uint64, C.c_int64, C.c_uint32, C.c_uint32]
        L.dpdo_philox_pair.restype = C.c_uint32
        L.dpdo_set_dt.argtypes = [vp, C.c_double]
        L.dpdo_set_pair.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, C.c_double]
        L.dpdo_renormalise_mom.argtypes = [vp]
        L.dpdo_set_slice_stress.argtypes = [vp, C.c_int32, C.c_int32, vp, C.c_int32, vp]
        L.dpdo_get_slice_stress.argtypes = [vp, vp, vp, vp]
        L.dpdo_slice_errors.argtypes = [vp]
        L.dpdo_slice_errors.restype = C.c_int64
        L.dpdo_random_state.argtypes = [C.c_int64, vp, C.c_double, C.c_uint64, C.c_int64, C.c_int64, vp, vp,
                                        vp, vp]
        L.dpdo_lamella_state.argtypes = [C.c_int64, vp, C.c_double, C.c_uint64, C.c_int64, C.c_int64, vp, vp,
                                         C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                         C.c_int32, C.c_double, C.c_int64, vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Oracle:
    """One oracle simulation of a DpdSystem (osprey_dpd_b200.workloads)."""

    def __init__(self, system, noise: int = NOISE_LCG, kT: float = None, gamma_scale: float = 1.0,
                 seed: int = None):
        L = lib()
        self._a = np.ascontiguousarray(system.a, dtype=np.float64)
        self._g = np.ascontiguousarray(system.gamma * gamma_scale, dtype=np.float64)
        seed = abs(int(system.seed if seed is None else seed))
        p = _Params(system.cells[0], system.cells[1], system.cells[2], *system.widths,
                    system.dt, system.lam, float(system.kT if kT is None else kT),
                    len(system.type_names), self._a.ctypes.data_as(C.POINTER(C.c_double)),
                    self._g.ctypes.data_as(C.POINTER(C.c_double)), seed, noise)
        self.h = L.dpdo_create(C.byref(p))
        if not self.h:
            raise RuntimeError("dpdo_create failed")
        self.n = system.n
        arrs = [np.ascontiguousarray(system.ids, np.int64), np.ascontiguousarray(system.types, np.int32),
                np.ascontiguousarray(system.movable, np.uint8), np.ascontiguousarray(system.x, np.float64),
                np.ascontiguousarray(system.unpbc, np.float64), np.ascontiguousarray(system.v, np.float64),
                np.ascontiguousarray(system.f, np.float64)]
        rc = L.dpdo_set_beads(self.h, self.n, *[_p(a) for a in arrs])
        if rc != 0:
            raise RuntimeError(f"dpdo_set_beads failed ({rc})")
        t = [np.ascontiguousarray(system.bond_head, np.int64), np.ascontiguousarray(system.bond_tail, np.int64),
             np.ascontiguousarray(system.bond_k2, np.float64), np.ascontiguousarray(system.bond_l0, np.float64),
             np.ascontiguousarray(system.angle_first, np.int64), np.ascontiguousarray(system.angle_second, np.int64),
             np.ascontiguousarray(system.angle_k3, np.float64), np.ascontiguousarray(system.angle_phi0, np.float64)]
        rc = L.dpdo_set_topology(self.h, len(t[0]), _p(t[0]), _p(t[1]), _p(t[2]), _p(t[3]),
                                 len(t[4]), _p(t[4]), _p(t[5]), _p(t[6]), _p(t[7]))
        if rc != 0:
            raise RuntimeError(f"dpdo_set_topology failed ({rc})")
        self._sys = system
        self._slices = 0

    def set_slice_stress(self, nslices: int) -> None:
        """Accumulates CMonitor's slice stress profile (Monitor.cpp:1900-2755)
        over ``nslices`` z slices every step; 0 turns it off."""
        s = self._sys
        self._bt = np.ascontiguousarray(s.bond_type if s.bond_type is not None else [], np.int32)
        self._at = np.ascontiguousarray(s.angle_type if s.angle_type is not None else [], np.int32)
        self._nbt = len(s.bond_specs)
        self._nbpt = len(s.bondpair_specs)
        rc = lib().dpdo_set_slice_stress(self.h, int(nslices), self._nbt, _p(self._bt), self._nbpt, _p(self._at))
        if rc != 0:
            raise RuntimeError(f"dpdo_set_slice_stress failed ({rc})")
        self._slices = int(nslices)

    def slice_stress(self):
        """{"pair": [S][T*T][9], "bond": [S][NBT][9], "bondpair": [S][NBPT][9]}
        of the last step."""
        S, T = self._slices, len(self._sys.type_names)
        out = {"pair": np.zeros((S, T * T, 9)), "bond": np.zeros((S, self._nbt, 9)),
               "bondpair": np.zeros((S, self._nbpt, 9))}
        if lib().dpdo_get_slice_stress(self.h, _p(out["pair"]), _p(out["bond"]), _p(out["bondpair"])) != 0:
            raise RuntimeError("slice stress is off")
        return out

    def slice_errors(self) -> int:
        return int(lib().dpdo_slice_errors(self.h))

    def step(self, first_step: int, nsteps: int) -> None:
        if lib().dpdo_step(self.h, first_step, nsteps) != 0:
            raise RuntimeError("dpdo_step failed")

    def state(self):
        n = self.n
        out = {k: np.zeros((n, 3)) for k in ("x", "unpbc", "v", "f")}
        out["stress"] = np.zeros((n, 9))
        lib().dpdo_get(self.h, _p(out["x"]), _p(out["unpbc"]), _p(out["v"]), _p(out["f"]), _p(out["stress"]))
        return out

    def cells(self) -> np.ndarray:
        c = np.zeros(self.n, dtype=np.int32)
        lib().dpdo_get_cells(self.h, _p(c))
        return c

    def cell_errors(self) -> int:
        return int(lib().dpdo_cell_errors(self.h))

    def pair_count(self) -> int:
        return int(lib().dpdo_pair_count(self.h))

    def set_dt(self, dt: float) -> None:
        lib().dpdo_set_dt(self.h, dt)

    def set_pair(self, ti: int, tj: int, a: float, gamma: float) -> None:
        lib().dpdo_set_pair(self.h, ti, tj, a, gamma)

    def renormalise_mom(self) -> None:
        """CSimBox::UpdateRenormalisedMom (SimBox.cpp:3177-3225)."""
        if lib().dpdo_renormalise_mom(self.h) != 0:
            raise RuntimeError("dpdo_renormalise_mom failed")

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().dpdo_destroy(h)
            self.h = None


def random_state(n: int, L, kT: float, seed: int, skip: int = 0, bond_head=None, bond_tail=None):
    """CRandomBuilder::Assemble restated (dpdo_random_state): (x, v), each
    (n, 3) in bead order, for ``n`` beads in a box of lengths ``L``; bonds as
    bead indices in the reference's polymer order."""
    x = np.zeros((n, 3))
    v = np.zeros((n, 3))
    Lv = np.ascontiguousarray(L, dtype=np.float64)
    bh = np.ascontiguousarray(bond_head if bond_head is not None else [], dtype=np.int64)
    bt = np.ascontiguousarray(bond_tail if bond_tail is not None else [], dtype=np.int64)
    rc = lib().dpdo_random_state(n, _p(Lv), kT, seed, skip, len(bh), _p(bh), _p(bt), _p(x), _p(v))
    if rc != 0:
        raise ValueError(f"bead {-1 - rc} drawn outside the box")
    return x, v


def lamella_state(L, kT: float, seed: int, poly_first, poly_type, lipid_type: int, head_offset: int,
                  tail_offset: int, normal: int = 2, centre: float = 0.5, thickness: float = 5.0,
                  linearise: bool = True, upper_fraction: float = 0.5, skip: int = 0, bond_head=None,
                  bond_tail=None):
    """CLamellaBuilder::Assemble restated (dpdo_lamella_state): (x, v), each
    (n, 3) in bead order; polymer p holds beads [poly_first[p],
    poly_first[p+1]); bonds as bead indices in polymer order."""
    pf = np.ascontiguousarray(poly_first, dtype=np.int64)
    pt = np.ascontiguousarray(poly_type, dtype=np.int32)
    n = int(pf[-1])
    x = np.zeros((n, 3))
    v = np.zeros((n, 3))
    Lv = np.ascontiguousarray(L, dtype=np.float64)
    bh = np.ascontiguousarray(bond_head if bond_head is not None else [], dtype=np.int64)
    bt = np.ascontiguousarray(bond_tail if bond_tail is not None else [], dtype=np.int64)
    rc = lib().dpdo_lamella_state(n, _p(Lv), kT, seed, skip, len(pt), _p(pf), _p(pt), lipid_type, head_offset,
                                  tail_offset, normal, centre, thickness, int(bool(linearise)), upper_fraction,
                                  len(bh), _p(bh), _p(bt), _p(x), _p(v))
    if rc != 0:
        raise ValueError({-1: "bad arguments", -2: "the bilayer does not fit the box",
                          -3: "lamella lattice outside the box"}.get(rc, str(rc)))
    return x, v


def philox_pair(seed: int, step: int, id_lo: int, id_hi: int) -> int:
    return int(lib().dpdo_philox_pair(seed, step, id_lo, id_hi))


def run_reference(system, steps: int, workdir: str = None, kT: float = None, gamma_scale: float = 1.0,
                  inject: bool = True, dump: bool = True, topology: bool = False, timeout: float = None,
                  rng_seed: int = None, slices: int = 0, initial: bool = False, paraview: bool = False,
                  state=None):
    """Runs the unmodified reference (oracle/_ref/osprey_ref_driver) on
    ``system`` for ``steps`` steps; ``rng_seed`` restarts its pair-noise LCG
    at that value just before the step loop; ``slices`` > 0 sets the analysis
    grid to that many z slices and also returns the last step's slice stress
    profile; ``initial`` adds the builder's state before any step as
    summary["initial"]; ``paraview`` the bytes of the reference's Paraview
    snapshot of the last step as summary["paraview"]; ``state`` the control
    file's initial-state block (workloads.lamella_block, default random).
    Returns (json summary, dump dict or None, topology dict or None)
    or, with ``slices``, (summary, dump, topology, slice dict)."""
    from osprey_dpd_b200 import workloads  # local import: test-side helper

    if not os.path.exists(REF_DRIVER):
        raise FileNotFoundError(REF_DRIVER)
    own = workdir is None
    wd = workdir or tempfile.mkdtemp(prefix="dpdref_")
    run = "r"
    workloads.write_dmpci(system, os.path.join(wd, "dmpci." + run), steps, kT=kT, gamma_scale=gamma_scale,
                          grid_z=max(1, int(slices)), state=state)
    args = [REF_DRIVER, run]
    if inject:
        workloads.write_state(system, os.path.join(wd, "state.bin"))
        args += ["--inject", "state.bin"]
    if dump:
        args += ["--dump", "out.bin"]
    if topology:
        args += ["--topology", "topo.bin"]
    if rng_seed is not None:
        args += ["--rng-seed", str(int(rng_seed))]
    if slices:
        dims = f"{int(slices)},{len(system.type_names)},{len(system.bond_specs)},{len(system.bondpair_specs)}"
        args += ["--slices", "slices.bin", "--slice-dims", dims]
    if initial:
        args += ["--dump-initial", "init.bin"]
    if paraview:
        args += ["--paraview", "1"]
    cp = subprocess.run(args, cwd=wd, capture_output=True, text=True, timeout=timeout)
    if cp.returncode != 0:
        raise RuntimeError(f"reference driver failed: {cp.stderr.strip()} {cp.stdout.strip()}")
    line = [l for l in cp.stdout.splitlines() if l.startswith("{")][-1]
    summary = json.loads(line)
    d = workloads.read_dump(os.path.join(wd, "out.bin")) if dump else None
    t = workloads.read_topology(os.path.join(wd, "topo.bin")) if topology else None
    sl = workloads.read_slices(os.path.join(wd, "slices.bin")) if slices else None
    if initial:
        summary["initial"] = workloads.read_dump(os.path.join(wd, "init.bin"))
    if paraview:
        vtk = [f for f in os.listdir(wd) if f.endswith(".vtk")]
        if len(vtk) != 1:
            raise RuntimeError(f"expected one Paraview file, found {vtk}")
        with open(os.path.join(wd, vtk[0]), "rb") as fh:
            summary["paraview"] = fh.read()
    if own:
        import shutil
        shutil.rmtree(wd, ignore_errors=True)
    return (summary, d, t, sl) if slices else (summary, d, t)
