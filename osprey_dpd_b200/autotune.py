"""Autotuner for the pair-force kernel's launch shape.

The shape of the force kernel (hit-list capacity per bead, persistent grid
or one tile per block, shared-memory carveout, and where the caller allows
run-to-run variation in the last bits, the half-shell pair scheme with its
tile of 64 or 128 beads per block) is chosen by timing candidate
shapes on the live workload: for each candidate the engine advances a scratch
copy of the system by a few captured multi-step calls and the fastest shape
wins.  Results are cached in a JSON file keyed by the GPU name and a
signature of the workload (bead count, cell count, bead types, precision,
number of boxes), so a run pays for tuning once.
"""
from __future__ import annotations

import json
import os
import time
from typing import Callable, Dict, Iterable, Optional, Tuple

Shape = Tuple[int, ...]     # (hitcap, persistent blocks per SM, carveout[, pair scheme[, half-shell tile]])

# full-shell shapes: bitwise reproducible forces
DEFAULT_CANDIDATES: Tuple[Shape, ...] = (
    (32, 0, -1), (40, 0, -1), (24, 0, -1), (48, 0, -1), (32, 0, 100), (32, 4, -1), (32, 8, -1),
)
# half-shell shapes (pair scheme 1): each pair once, atomics, last bits vary;
# tiles of 64 (two warps) and 128 beads (four warps) per block
HALF_SHELL_CANDIDATES: Tuple[Shape, ...] = (
    (32, 0, -1, 1, 64), (24, 0, -1, 1, 64), (32, 0, 100, 1, 64), (24, 0, 100, 1, 64), (40, 0, 100, 1, 64),
    (32, 0, -1, 1, 128), (24, 0, 100, 1, 128),
)
# staged half-shell shape (pair scheme 2): smaller hit lists leave room for the staged rows
STAGED_CANDIDATES: Tuple[Shape, ...] = ((16, 0, 100, 2),)
CACHE = os.environ.get("DPD_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "osprey_dpd_b200",
                                                       "launch_shapes.json"))


def signature(gpu: str, n: int, ncells: int, ntypes: int, precision: int, nboxes: int,
              reproducible: bool = True) -> str:
    sig = f"{gpu}|n={n}|cells={ncells}|types={ntypes}|prec={precision}|boxes={nboxes}"
    return sig if reproducible else sig + "|half"


def apply_shape(eng, shape: Shape) -> None:
    """Sets a tuned shape on an engine (the scheme and the half-shell tile only
    when the shape names them)."""
    eng.set_launch_shape(*shape[:3])
    if len(shape) > 3:
        eng.set_pair_scheme(shape[3])
    if len(shape) > 4:
        eng.set_pair_tile(shape[4])


def _load(path: str) -> Dict[str, dict]:
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(path: str, table: Dict[str, dict]) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune(make_engine: Callable[[], object], sig: str, candidates: Iterable[Shape] = DEFAULT_CANDIDATES,
         steps: int = 20, reps: int = 3, sync: Optional[Callable[[], None]] = None,
         cache_path: str = CACHE, force: bool = False) -> dict:
    """Times every candidate shape on a fresh engine from ``make_engine`` and
    returns {"shape": best, "ms_per_step": ..., "trials": {...}}; cached by sig."""
    table = _load(cache_path)
    if not force and sig in table:
        return table[sig]
    trials = {}
    for shape in candidates:
        eng = make_engine()
        apply_shape(eng, shape)
        t = 1
        eng.step(t, steps)       # capture + warm-up
        t += steps
        eng.status()
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            eng.step(t, steps)
            eng.status()         # waits for the work
            best = min(best, (time.perf_counter() - t0) * 1000.0 / steps)
            t += steps
        eng.close()
        trials[",".join(map(str, shape))] = best
    win = min(trials, key=trials.get)
    res = {"shape": [int(v) for v in win.split(",")], "ms_per_step": trials[win], "trials": trials}
    table[sig] = res
    _store(cache_path, table)
    return res
