"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names.update(re.findall(r"DPD_API\s+[\w\s\*]+?\b(\w+)\s*\(", src))
    return sorted(names)


def test_headers_declare_entry_points():
    syms = declared_symbols()
    assert "dpd_engine_create" in syms and "dpd_engine_step" in syms
    assert len(syms) >= 15


def test_library_exports_every_declared_symbol():
    from osprey_dpd_b200 import build, engine
    lib = build.build()
    dll = ctypes.CDLL(lib)
    missing = [s for s in declared_symbols() if not hasattr(dll, s)]
    assert not missing, missing
    engine.load()   # argtypes for every binding resolve
    assert set(engine.EXPORTED) <= set(declared_symbols())


def test_create_rejects_bad_parameters_without_gpu_work():
    from osprey_dpd_b200 import engine
    L = engine.load()
    h = ctypes.c_void_p()
    # nx < 3 is rejected before any CUDA call
    import numpy as np
    a = np.array([[25.0]])
    g = np.array([[4.5]])
    p = engine.DpdParams(2, 10, 10, 1.0, 1.0, 1.0, 0.02, 0.5, 1.0, 1,
                         a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                         g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1, 0, -1)
    assert L.dpd_engine_create(ctypes.byref(p), ctypes.byref(h)) == -1
    assert not h.value
