"""Builds the engine's shared library for sm_100a with nvcc (no JIT cache):
osprey_dpd_b200/_build/libospreydpd_cuda.so."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libospreydpd_cuda.so")
SOURCES = [os.path.join(HERE, "csrc", "dpd_engine.cu"), os.path.join(HERE, "csrc", "dpd_noalloc.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))] + \
    [os.path.join(ROOT, "include", "dpd_engine.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-shared",
              "-Xptxas", "-v", "-cudart", "static"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB + ".tmp"] + SOURCES
    cp = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(BUILD, "ptxas.log")
    with open(log, "w") as fh:
        fh.write(" ".join(cmd) + "\n" + cp.stdout + cp.stderr)
    if cp.returncode != 0:
        sys.stderr.write(cp.stderr)
        raise RuntimeError("nvcc failed for the DPD engine; see " + log)
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        sys.stdout.write(cp.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
