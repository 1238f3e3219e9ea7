"""The allocation-free pair-force entry point (dpd_pair_forces_noalloc).

It serves callers that may not allocate device memory when they need forces
(a host whose memory pool owns the GPU, capture-sensitive or real-time loops,
plug-ins whose host forbids library allocations): they pass their own device
buffers and the cell-list scratch comes from a fixed array inside the
library.  The check: its forces equal the engine's own first-step pair forces
(through dpd_engine_*) within the mixed-precision force tolerance of the other
parity tests, on two calls in a row (the second call must not see leftovers
of the first).  This file sorts last so a run that stops at the first failure
has already run every other test.
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


def test_noalloc_matches_engine_forces_twice(engine_mod):
    import torch
    s = W.binary_mixture(cells=(16, 17, 18), a_ab=40.0)       # 14,688 beads, no bonds
    s.f[:] = 0.0          # so the first step's intermediate velocity equals v0
    eng = engine_mod.DpdEngine.from_system(s, precision=engine_mod.MIXED, device=0)
    eng.step(1, 1)
    ref = eng.download()
    assert eng.status() == 0
    eng.close()

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
    assert np.array_equal(outs[0], outs[1])


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
