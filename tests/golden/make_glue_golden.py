"""Reference results for the engine binding's end-to-end runs.

Runs the reference's own program (oracle/_ref/osprey_ref_main: its dmpc.cpp
main over objects compiled from its src/*.cpp) on the control files in
tests/golden/dmpci/ and keeps the time series of its history file
(dmpchs.<runId>: sample time, temperature, pressure, ... as CMonitor writes
them), so the GPU tests can compare the engine binding's own history files
with the reference's statistics.  Written to tests/golden/glue_<name>.npz:

    python tests/golden/make_glue_golden.py
"""
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "osprey_ref_main")
RUNS = ("water", "bilayer")


def read_history(path):
    rows = [list(map(float, ln.split())) for ln in open(path) if ln.strip()]
    if not rows:
        return None   # a run stopped before its first sample
    width = min(len(r) for r in rows)
    return np.array([r[:width] for r in rows])


def run(program, name, env=None, timeout=1800):
    """Runs `program` on tests/golden/dmpci/dmpci.<name> in a scratch
    directory; returns (history array, log text, seconds)."""
    d = tempfile.mkdtemp(prefix=f"dpd_{name}_")
    try:
        shutil.copy(os.path.join(HERE, "dmpci", f"dmpci.{name}"), os.path.join(d, f"dmpci.{name}"))
        t0 = time.perf_counter()
        cp = subprocess.run([program, name], cwd=d, capture_output=True, text=True, timeout=timeout,
                            env=dict(os.environ, **(env or {})))
        dt = time.perf_counter() - t0
        if cp.returncode != 0:
            raise RuntimeError(f"{program} {name}: exit {cp.returncode}\n{cp.stdout}\n{cp.stderr}")
        log = open(os.path.join(d, f"dmpcls.{name}")).read() if os.path.exists(os.path.join(d, f"dmpcls.{name}")) else ""
        hist = os.path.join(d, f"dmpchs.{name}")
        return (read_history(hist) if os.path.exists(hist) else None), log, dt
    finally:
        shutil.rmtree(d, ignore_errors=True)


def main():
    for name in (sys.argv[1:] or RUNS):
        hist, log, dt = run(REF_MAIN, name)
        np.savez_compressed(os.path.join(HERE, f"glue_{name}.npz"), history=hist, seconds=dt)
        print(name, hist.shape, f"{dt:.1f} s")


if __name__ == "__main__":
    main()
