"""The allocation-free pair-force entry point (dpd_pair_forces_noalloc).

It serves callers that may not allocate device memory when they need forces
(a host whose memory pool owns the GPU, real-time loops, plug-ins whose host
forbids library allocations): they pass their own device buffers and the
cell-list scratch comes from a fixed array inside the library.  The check:
its forces equal the engine's own first-step pair forces (through
dpd_engine_*) and the CPU oracle's, within the mixed-precision force
tolerance of the other parity tests, on two calls in a row (the second call
must not see leftovers of the first).  Error cases: sizes beyond the
scratch, a bead outside the box, bad parameters and bead types.  This file
sorts last so a run that stops at the first failure has already run every
other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORCE_TOL_MIXED = 1e-5      # same bound as the engine's mixed-precision parity tests


def _bind(engine_mod):
    L = engine_mod.load()
    fn = L.dpd_pair_forces_noalloc
    fn.argtypes = [C.POINTER(engine_mod.DpdParams), C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _params(engine_mod, s, a, g):
    return engine_mod.DpdParams(s.cells[0], s.cells[1], s.cells[2], *s.widths, s.dt, s.lam, s.kT,
                                a.shape[0], a.ctypes.data_as(C.POINTER(C.c_double)),
                                g.ctypes.data_as(C.POINTER(C.c_double)), abs(int(s.seed)), 0, 0)


def test_noalloc_matches_engine_forces_twice(engine_mod, oracle_mod):
    import torch
    s = W.binary_mixture(cells=(16, 17, 18), a_ab=40.0)       # 14,688 beads, no bonds
    s.f[:] = 0.0          # so the first step's intermediate velocity equals v0
    eng = engine_mod.DpdEngine.from_system(s, precision=engine_mod.MIXED, device=0)
    eng.step(1, 1)
    ref = eng.download()
    assert eng.status() == 0
    eng.close()
    # the CPU oracle (the reference's algorithm, same Philox pair noise) on the same first step
    orc = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    orc.step(1, 1)
    ora = orc.state()
    assert np.array_equal(ora["x"], ref["x"])

    dev = torch.device("cuda", 0)
    x = torch.from_numpy(np.ascontiguousarray(ref["x"])).to(dev)
    v = torch.from_numpy(np.ascontiguousarray(s.v)).to(dev)
    t = torch.from_numpy(s.types.astype(np.int32)).to(dev)
    i = torch.from_numpy(s.ids.astype(np.int32)).to(dev)
    a = np.ascontiguousarray(s.a)
    g = np.ascontiguousarray(s.gamma)
    p = _params(engine_mod, s, a, g)
    fn = _bind(engine_mod)
    outs = []
    for _ in range(2):
        f = torch.full((s.n, 3), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = fn(C.byref(p), 1, s.n, x.data_ptr(), v.data_ptr(), t.data_ptr(), i.data_ptr(), f.data_ptr(), None)
        assert rc == 0
        outs.append(f.cpu().numpy())
    for out in outs:
        assert np.all(np.isfinite(out))
        assert rel_err(out, ref["f"]) < FORCE_TOL_MIXED
        assert rel_err(out, ora["f"]) < FORCE_TOL_MIXED
    assert np.array_equal(outs[0], outs[1])


def _device_inputs(s, x):
    import torch
    dev = torch.device("cuda", 0)
    return (torch.from_numpy(np.ascontiguousarray(x)).to(dev), torch.from_numpy(np.ascontiguousarray(s.v)).to(dev),
            torch.from_numpy(s.types.astype(np.int32)).to(dev), torch.from_numpy(s.ids.astype(np.int32)).to(dev),
            torch.zeros((s.n, 3), dtype=torch.float64, device=dev))


def test_noalloc_reports_a_bead_outside_the_box(engine_mod):
    """A bead at x = L is outside the reference's cells: DPD_E_BOX, finite output."""
    import torch
    s = W.water(10)
    x = s.x.copy()
    x[17, 0] = s.cells[0] * s.widths[0]
    xd, vd, td, idd, fd = _device_inputs(s, x)
    a, g = np.ascontiguousarray(s.a), np.ascontiguousarray(s.gamma)
    p = _params(engine_mod, s, a, g)
    fn = _bind(engine_mod)
    torch.cuda.synchronize()
    assert fn(C.byref(p), 1, s.n, xd.data_ptr(), vd.data_ptr(), td.data_ptr(), idd.data_ptr(), fd.data_ptr(),
              None) == -4
    assert np.all(np.isfinite(fd.cpu().numpy()))


def test_noalloc_rejects_bad_parameters_and_types(engine_mod):
    import torch
    s = W.binary_mixture(cells=(8, 8, 8))
    a, g = np.ascontiguousarray(s.a), np.ascontiguousarray(s.gamma)
    fn = _bind(engine_mod)
    # ntypes above the pair tables' capacity: rejected on the host
    p = _params(engine_mod, s, a, g)
    p.ntypes = 33
    assert fn(C.byref(p), 1, s.n, 1, 1, 1, 1, 1, None) == -1
    # a bead type outside 0..ntypes-1: found on the device, DPD_E_ARG
    types = s.types.astype(np.int32).copy()
    types[5] = 2
    xd, vd, _, idd, fd = _device_inputs(s, s.x)
    td = torch.from_numpy(types).to(xd.device)
    p = _params(engine_mod, s, a, g)
    torch.cuda.synchronize()
    assert fn(C.byref(p), 1, s.n, xd.data_ptr(), vd.data_ptr(), td.data_ptr(), idd.data_ptr(), fd.data_ptr(),
              None) == -1
    # and the next good call is unaffected by the bad one
    td = torch.from_numpy(s.types.astype(np.int32)).to(xd.device)
    assert fn(C.byref(p), 1, s.n, xd.data_ptr(), vd.data_ptr(), td.data_ptr(), idd.data_ptr(), fd.data_ptr(),
              None) == 0


def test_noalloc_rejects_sizes_beyond_its_scratch(engine_mod):
    s = W.water(10)
    a = np.ascontiguousarray(s.a)
    g = np.ascontiguousarray(s.gamma)
    p = _params(engine_mod, s, a, g)
    fn = _bind(engine_mod)
    # too many beads: rejected before any pointer is touched
    assert fn(C.byref(p), 1, 65537, 1, 1, 1, 1, 1, None) == -7
    # too many cells
    p.nx, p.ny, p.nz = 40, 40, 40
    assert fn(C.byref(p), 1, 100, 1, 1, 1, 1, 1, None) == -7
