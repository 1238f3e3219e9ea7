#!/usr/bin/env python
"""DPD step throughput on one or more B200s, in bead-steps/s.

Workload (default): the H3T6 lipid bilayer in water, 64x64x32 cells of unit
width at density 3 -> 393,216 beads, 6,000 lipids (48,000 bonds, 24,000 tail
bond pairs), a_ij of the reference's bilayer example, gamma = 4.5, kT = 1,
dt = 0.02.  Synthetic, seeded (osprey_dpd_b200/workloads.py).

A step is one full DPD timestep (UpdatePos, cell re-binning, pair forces,
bond + bond-pair forces, UpdateMom).  `value` is the mixed-precision
(FP32 forces, FP64 positions/velocities/sums) throughput with the state
resident in HBM; the all-FP64 form is timed the same way.  L2 is flushed before
every timed step (a 256 MiB write, then a 256 MiB read of another buffer so
that the write's dirty lines are back in HBM), each step is timed with CUDA
events on the engine's stream, and the max over ranks is reported.  `e2e` is the same
metric through the C ABI with host buffers: upload the bead state, run one
reference sample period (100 steps), read back the single-bead sums and the
full bead state.

`--impl reference` times the reference itself: Osprey-DPD's own serial step
loop, compiled from its sources (oracle/_ref), on the host cores.

Multi-GPU (torchrun): every rank advances its own replica of the workload
(weak scaling; no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "bead-steps/s, 393k-bead bilayer: FP32/FP64-mixed vs all-FP64, 1 B200"
REPLICA_METRIC = "bead-steps/s, 512-replica A/B sweep: one batch vs replicas one at a time, 1 B200"
UNIT = "bead-steps/s"
SAMPLE_PERIOD = 100       # SamplePeriod of the reference's bilayer example (examples/dmpci.bilayer)
E2E_PERIOD = SAMPLE_PERIOD
L2_FLUSH_BYTES = 256 << 20
SLOTS_PER_BEAD_STEP = 755.0   # pair-force issue work per bead-step (half shell, rho = 3)
ALG_BYTES_PER_BEAD_STEP = {"mixed": 124.0, "fp64": 148.0}   # whole-step algorithmic HBM bytes


def workload(name: str, seed_offset: int = 0):
    from osprey_dpd_b200 import workloads as W
    if name == "bilayer":
        s = W.bilayer(seed=W.BASE_SEED + 3 + 7919 * seed_offset)
        desc = "H3T6 bilayer in water, 64x64x32 cells, 393,216 beads, 6,000 lipids"
    elif name == "water":
        s = W.water(10, seed=W.BASE_SEED + 1 + 7919 * seed_offset)
        desc = "DPD water 10x10x10, 3,000 beads"
    elif name == "binary":
        s = W.binary_mixture(32, seed=W.BASE_SEED + 2 + 7919 * seed_offset)
        desc = "A/B mixture 32^3, 98,304 beads, a_AB = 50"
    elif name == "polymer":
        s = W.polymer_solution(128, seed=W.BASE_SEED + 4 + 7919 * seed_offset)
        desc = "16-bead chains (30%) in solvent, 128^3, 6,291,456 beads"
    else:
        raise SystemExit(f"unknown workload {name}")
    return s, desc


def dist_info():
    from osprey_dpd_b200 import ranks
    return ranks.layout()


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_sample(system, steps: int, timeout: float = 600.0) -> dict:
    """Times the reference's own step loop (oracle/_ref): two runs from the
    same state, of steps // 3 and `steps` steps, differenced, so that what
    CSimBox::Run spends once (about 4 s before the first step of the
    393k-bead bilayer on a container core, 0.8 s a step after it) cancels
    and the rate is the loop's steady one.  run_seconds and steps are those
    of the difference."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dpd_oracle
    if os.path.exists(dpd_oracle.REF_DRIVER):
        steps = max(2, steps)
        short = max(1, steps // 3)
        s_short, _, _ = dpd_oracle.run_reference(system, short, dump=False, timeout=timeout)
        s_long, _, _ = dpd_oracle.run_reference(system, steps, dump=False, timeout=timeout)
        dt = s_long["run_seconds"] - s_short["run_seconds"]
        diff = steps - short
        if dt <= 0.0:   # timing noise larger than the difference: the long run alone
            dt, diff = s_long["run_seconds"], steps
        return {"value": system.n * diff / dt, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"{steps} minus {short} steps of the full {system.n}-bead workload, reference step loop "
                          f"(CSimBox::Run) timed without set-up and differenced, 1 thread",
                "run_seconds": dt, "steps": diff}
    o = dpd_oracle.Oracle(system)
    t0 = time.perf_counter()
    o.step(1, steps)
    dt = time.perf_counter() - t0
    return {"value": system.n * steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{steps} steps of the full {system.n}-bead workload, C restatement, 1 thread",
            "run_seconds": dt, "steps": steps}


def reference_replica_aggregate(nrep: int, cores: int, seconds: float = 15.0) -> dict:
    """The reference on the replica sweep with all host cores: the first
    min(cores, nrep) replicas run at once, one reference process each, every
    process for about `seconds` of its own step loop; the aggregate is the sum
    of the processes' bead-steps/s (each measured while the others run)."""
    from concurrent.futures import ThreadPoolExecutor
    from osprey_dpd_b200 import workloads as W
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dpd_oracle
    if not os.path.exists(dpd_oracle.REF_DRIVER):
        raise FileNotFoundError(dpd_oracle.REF_DRIVER)
    p = max(1, min(cores, nrep))
    systems = [W.replica(r, nrep) for r in range(p)]
    steps = [max(5, min(2000, int(seconds * 5e5 / s.n))) for s in systems]

    def one(k):
        summary, _, _ = dpd_oracle.run_reference(systems[k], steps[k], dump=False, timeout=20 * seconds + 300)
        return summary["bead_steps_per_s"], summary["run_seconds"]

    with ThreadPoolExecutor(max_workers=p) as pool:
        res = list(pool.map(one, range(p)))
    agg = sum(r[0] for r in res)
    return {"value": agg, "unit": UNIT, "cores": p, "kind": "reference",
            "sample": f"replicas 0..{p - 1} of {nrep} ({sum(s.n for s in systems)} beads), one reference process "
                      f"each, {min(steps)}-{max(steps)} steps, run at once; sum of the processes' rates",
            "run_seconds": max(r[1] for r in res)}


def run_reference_arm(args):
    ws, rank, _ = dist_info()
    if rank != 0:
        return 0
    if args.workload == "replicas":
        cb = reference_replica_aggregate(args.replicas, os.cpu_count() or 1)
        line = {"impl": "reference", "metric": REPLICA_METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded replica table)",
                "config": {"workload": f"{args.replicas} A/B replicas, edges 8..24 (all-cores sample)",
                           "precision": "reference FP64"},
                "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    system, desc = workload(args.workload)
    # bounded sample: two runs (a third and all of `steps`) within about a
    # minute of the serial reference
    per_step_est = system.n / 0.5e6
    steps = max(2, min(args.steps, int(45.0 / per_step_est)))
    cb = cpu_reference_sample(system, steps)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": ws,
            "steps": cb["steps"], "warmup": args.warmup, "ms_per_step": 1000.0 * cb["run_seconds"] / cb["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": desc, "n_beads": system.n,
                                                     "precision": "reference FP64"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def tune_candidates(reproducible: bool):
    from osprey_dpd_b200 import autotune
    if reproducible:
        return autotune.DEFAULT_CANDIDATES
    return autotune.DEFAULT_CANDIDATES + autotune.HALF_SHELL_CANDIDATES + autotune.STAGED_CANDIDATES


# default shape per scheme (half shell: hit lists of 24 and two-warp tiles, the
# autotuner's choice on the bilayer and the fastest capacity on the melt)
FIXED_SHAPES = {"full": (32, 0, -1, 0), "half": (24, 0, -1, 1, 64), "staged": (16, 0, 100, 2)}
SCHEME_NAMES = {0: "full", 1: "half", 2: "staged"}
PAIR_KERNELS = {"full": "k_pair_forces", "half": "k_pair_forces_half", "staged": "k_pair_forces_staged"}


def tuned_shape(engine_mod, system, precision: int, dev, torch, enabled: bool, reproducible: bool = False,
                scheme: str = "auto"):
    """Pair-kernel launch shape from the autotuner (cached per GPU and workload),
    or the default shape of a fixed scheme."""
    if scheme != "auto":
        return {"shape": list(FIXED_SHAPES[scheme])}
    if not enabled:
        return None
    from osprey_dpd_b200 import autotune
    sig = autotune.signature(torch.cuda.get_device_name(dev), system.n, system.ncells, len(system.type_names),
                             precision, 1, reproducible)
    make = lambda: engine_mod.DpdEngine.from_system(system, precision=precision, device=dev.index)
    return autotune.tune(make, sig, tune_candidates(reproducible), steps=10, reps=2)


def scheme_of(shape) -> str:
    return SCHEME_NAMES[shape[3]] if shape and len(shape) > 3 else "full"


def pair_scheme_name(shape) -> str:
    return {"full": "full shell (reproducible)", "half": "half shell (atomics)",
            "staged": "half shell staged in shared memory (atomics)"}[scheme_of(shape)]


def time_engine(engine_mod, system, precision: int, steps: int, warmup: int, dev, torch, profile: bool,
                shape=None, profile_steps: int = 20, flush: bool = True):
    """Per-step device time (ms) of single-step calls with L2 flushed before
    each step; then, when asked, a separate pass with CUDA events around every
    kernel (launched one by one) for the per-kernel durations."""
    from osprey_dpd_b200 import autotune
    eng = engine_mod.DpdEngine.from_system(system, precision=precision, device=dev.index)
    if shape:
        autotune.apply_shape(eng, shape)
    eng.set_sample_period(SAMPLE_PERIOD)
    stream = torch.cuda.Stream(device=dev)
    eng.set_stream(stream.cuda_stream)
    flush_buf = torch.empty(L2_FLUSH_BYTES if flush else 1, dtype=torch.uint8, device=dev)
    clean = torch.ones(L2_FLUSH_BYTES // 4 if flush else 1, dtype=torch.float32, device=dev)

    def flush_l2():
        # evict the state by writing a buffer larger than L2, then read a second
        # one so the dirty lines of the first are written back before the step
        if not flush:
            return None
        flush_buf.zero_()
        return clean.sum()

    t = 1
    for _ in range(warmup):
        with torch.cuda.stream(stream):
            flush_l2()
        eng.step(t, 1)
        t += 1
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    launches0 = eng.launch_count()
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush_l2()
            evs[k][0].record(stream)
        eng.step(t, 1)
        with torch.cuda.stream(stream):
            evs[k][1].record(stream)
        t += 1
    torch.cuda.synchronize(dev)
    launches = eng.launch_count() - launches0
    ms = [a.elapsed_time(b) for a, b in evs]
    prof = None
    if profile:
        eng.profile(True)
        for _ in range(profile_steps):
            with torch.cuda.stream(stream):
                flush_l2()
            eng.step(t, 1)
            t += 1
        torch.cuda.synchronize(dev)
        prof = eng.profile_read()
        eng.profile(False)
    status = eng.status()
    eng.close()
    return ms, prof, launches, status


def e2e_run(engine_mod, system, precision: int, reps: int, dev, torch, shape=None):
    """Reference-facing call sequence with host buffers: upload, one sample
    period of steps, single-bead sums and the full state back to the host."""
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    ids, types, mov = pin(system.ids), pin(system.types), pin(system.movable)
    x, u, v, f = pin(system.x), pin(system.unpbc), pin(system.v), pin(system.f)
    out = {k: torch.empty((system.n, 3), dtype=torch.float64).pin_memory().numpy() for k in ("x", "u", "v", "f")}
    eng = engine_mod.DpdEngine(system.cells, system.widths, system.dt, system.lam, system.kT, system.a,
                               system.gamma, abs(int(system.seed)), precision, dev.index)
    if shape:
        from osprey_dpd_b200 import autotune
        autotune.apply_shape(eng, shape)
    h2d = ids.nbytes + types.nbytes + mov.nbytes + x.nbytes + u.nbytes + v.nbytes + f.nbytes
    d2h = sum(a.nbytes for a in out.values()) + 8 * 23
    times = []
    t = 1
    for r in range(reps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        eng.upload_beads(ids, types, mov, x, u, v, f)
        eng.upload_topology(system.bond_head, system.bond_tail, system.bond_k2, system.bond_l0,
                            system.angle_first, system.angle_second, system.angle_k3, system.angle_phi0)
        eng.step(t, E2E_PERIOD)
        eng.observables()
        eng.download_into(out["x"], out["u"], out["v"], out["f"])
        t1 = time.perf_counter()
        if r > 0:           # the first call also pays library/context start-up
            times.append(t1 - t0)
        t += E2E_PERIOD
    eng.close()
    topo_bytes = (system.bond_head.nbytes * 2 + system.bond_k2.nbytes * 2 +
                  system.angle_first.nbytes * 2 + system.angle_k3.nbytes * 2)
    return times, (h2d + topo_bytes) / E2E_PERIOD, d2h / E2E_PERIOD


def run_slab_exchange(args, dev, torch):
    """The device slab engine on one GPU: the workload split into
    args.slab_exchange z-slabs, every slab held by this process
    (DeviceSlabs.step_local, buffers swapped by device copies).  Wall clock
    per phase with the slabs' streams drained in between: the steps of all
    slabs, the pack, the buffer swap and the unpack (next local box, upload,
    topology filter); the whole box in one engine beside it (single-step
    calls).  On several GPUs the slabs' steps and exchanges run concurrently;
    this measures what one exchange costs, not a scaling curve."""
    import time
    from osprey_dpd_b200 import engine as E, slabs as S
    system, desc = workload(args.workload)
    prec = E.FP64 if args.precision == "fp64" else E.MIXED
    scheme = {"full": E.PAIR_FULL_SHELL, "staged": E.PAIR_STAGED}.get(args.pair_scheme, E.PAIR_HALF_SHELL)
    W = args.slab_exchange
    dn = dev.index
    e = E.DpdEngine.from_system(system, precision=prec, device=dn)
    e.set_pair_scheme(scheme)
    e.step(1, args.warmup)
    e.status()
    t0 = time.perf_counter()
    for t in range(args.warmup + 1, args.warmup + 1 + args.steps):
        e.step(t, 1)
    e.status()
    single = (time.perf_counter() - t0) / args.steps * 1e3
    e.close()
    sl = [S.DeviceSlabs(system, None, device=dn, rank=r, world=W, precision=prec, pair_scheme=scheme)
          for r in range(W)]
    S.DeviceSlabs.exchange_local(sl)
    for t in range(1, args.warmup + 1):
        S.DeviceSlabs.step_local(sl, t)
    ph = {"steps": 0.0, "pack": 0.0, "swap": 0.0, "unpack": 0.0}

    def drain():
        for x in sl:
            x.stream.synchronize()

    for t in range(args.warmup + 1, args.warmup + 1 + args.steps):
        a = time.perf_counter()
        for x in sl:
            x.eng.step(t, 1)
        drain()
        b = time.perf_counter()
        for x in sl:
            x.pack()
        drain()
        c = time.perf_counter()
        for r, x in enumerate(sl):
            with torch.cuda.stream(x.stream):
                x.bufs[2].copy_(sl[(r - 1) % W].bufs[1])
                x.bufs[3].copy_(sl[(r + 1) % W].bufs[0])
        drain()
        d = time.perf_counter()
        for x in sl:
            x.unpack()
        drain()
        f = time.perf_counter()
        ph["steps"] += b - a
        ph["pack"] += c - b
        ph["swap"] += d - c
        ph["unpack"] += f - d
    status = [x.eng.status() for x in sl]
    owned = sum(x.n_owned for x in sl)
    local = [x.n_local for x in sl]
    for x in sl:
        x.close()
    ms = {k: v / args.steps * 1e3 for k, v in ph.items()}
    return {"metric": "device slab engine on one GPU: ms per step and per exchange, all slabs together",
            "impl": "slab_exchange", "config": {"workload": desc, "slabs": W, "ghost_layers": 2,
                                                "precision": args.precision if args.precision != "both" else "mixed",
                                                "pair_scheme": pair_scheme_name((0, 0, 0, scheme))},
            "steps": args.steps, "warmup": args.warmup, "single_box_ms_per_step": single,
            "slabs_ms": ms, "exchange_ms": ms["pack"] + ms["swap"] + ms["unpack"],
            "owned_beads": owned, "local_beads": local, "status_bits": status,
            "timing": "wall clock per phase, every slab's stream drained between phases; one process, one GPU"}


def run_replica_sweep(args, dev, torch, E):
    """512 independent A/B replicas (box edges 8..24, A fraction 0.1..0.5,
    a_AB 25 -> 60, own seeds): one batch advanced as a captured 100-step CUDA
    graph, against the same replicas stepped one engine at a time (each also
    replaying its own 100-step graph).  The state (~1 GB) exceeds L2."""
    from osprey_dpd_b200 import workloads as W
    nrep = args.replicas
    systems = [W.replica(r, nrep) for r in range(nrep)]
    ntot = sum(s.n for s in systems)
    K = args.graph_steps
    stream = torch.cuda.Stream(device=dev)
    shape = list(FIXED_SHAPES[args.pair_scheme]) if args.pair_scheme != "auto" else None
    from osprey_dpd_b200 import autotune
    if shape is None and not args.no_autotune:
        sig = autotune.signature(torch.cuda.get_device_name(dev), ntot, sum(s.ncells for s in systems), 2, 0, nrep,
                                 args.reproducible)
        shape = autotune.tune(lambda: E.DpdBatch(systems, precision=E.MIXED, device=dev.index), sig,
                              tune_candidates(args.reproducible), steps=K, reps=1)["shape"]
    batch = E.DpdBatch(systems, precision=E.MIXED, device=dev.index)
    if shape:
        autotune.apply_shape(batch, shape)
    batch.set_sample_period(K)
    batch.set_stream(stream.cuda_stream)
    t = 1
    for _ in range(args.warmup):
        batch.step(t, K)
        t += K
    torch.cuda.synchronize(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    l0 = batch.launch_count()
    with torch.cuda.stream(stream):
        ev[0].record(stream)
    for _ in range(args.steps):
        batch.step(t, K)
        t += K
    with torch.cuda.stream(stream):
        ev[1].record(stream)
    torch.cuda.synchronize(dev)
    batch_ms = ev[0].elapsed_time(ev[1])
    batch_launches = batch.launch_count() - l0
    batch_status = batch.status()
    batch.close()
    # one at a time
    engines = []
    for s in systems:
        e = E.DpdEngine.from_system(s, precision=E.MIXED, device=dev.index, topology=False)
        if shape:     # the same pair scheme; the batch's tuned shape
            autotune.apply_shape(e, shape)
        e.set_sample_period(K)
        e.set_stream(stream.cuda_stream)
        engines.append(e)
    t = 1
    for _ in range(args.warmup):
        for e in engines:
            e.step(t, K)
        t += K
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(stream):
        ev[0].record(stream)
    for _ in range(args.steps):
        for e in engines:
            e.step(t, K)
        t += K
    with torch.cuda.stream(stream):
        ev[1].record(stream)
    torch.cuda.synchronize(dev)
    single_ms = ev[0].elapsed_time(ev[1])
    for e in engines:
        e.close()
    work = ntot * K * args.steps
    return {
        "metric": REPLICA_METRIC,
        "value": work / (batch_ms / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": args.steps * K,
        "warmup": args.warmup * K, "ms_per_step": batch_ms / (args.steps * K), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 forces / f64 state",
        "data": "synthetic (seeded replica table)",
        "config": {"workload": f"{nrep} A/B replicas, edges 8..24, {ntot} beads in total", "n_beads": ntot,
                   "graph_steps": K, "l2": "state (~1 GB) larger than L2", "precision": "mixed",
                   "pair_scheme": pair_scheme_name(shape)},
        "one_at_a_time": {"value": work / (single_ms / 1000.0), "ms_per_step": single_ms / (args.steps * K)},
        "batch_over_one_at_a_time": single_ms / batch_ms,
        "gpu_launches": batch_launches, "status_bits": batch_status, "launch_shape": shape,
    }


def time_melt(engine_mod, dev, torch, warmup: int, steps: int = 20):
    """The 6,291,456-bead polymer solution (target: >= 1.5e9 bead-steps/s),
    mixed precision, the half-shell scheme: per-step CUDA-event times
    of single-step calls; its state (~1.3 GB) exceeds L2, so no flush."""
    system, desc = workload("polymer")
    ms, prof, launches, status = time_engine(engine_mod, system, engine_mod.MIXED, steps, warmup, dev, torch, False,
                                             list(FIXED_SHAPES["half"]), flush=False)
    total = sum(ms)
    return {"workload": desc, "n_beads": system.n, "value": system.n * steps / (total / 1000.0),
            "unit": UNIT, "ms_per_step": total / steps, "steps": steps, "warmup": warmup, "target": 1.5e9,
            "precision": "mixed", "pair_scheme": pair_scheme_name(FIXED_SHAPES["half"]),
            "l2": "state (~1.3 GB) larger than L2", "gpu_launches": launches, "status_bits": status}


def time_sweep(engine_mod, dev, torch, nrep: int = 512, graph_steps: int = 100):
    """The 512-replica A/B sweep (target: >= 3x over the replicas one at a
    time): one batch of all replicas as captured 100-step graphs against the
    same replicas stepped engine by engine, one 100-step call each."""
    ns = argparse.Namespace(replicas=nrep, graph_steps=graph_steps, steps=1, warmup=1, pair_scheme="half",
                            no_autotune=True, reproducible=False)
    r = run_replica_sweep(ns, dev, torch, engine_mod)
    return {"workload": r["config"]["workload"], "value": r["value"], "unit": UNIT,
            "ms_per_step": r["ms_per_step"], "one_at_a_time": r["one_at_a_time"],
            "batch_over_one_at_a_time": r["batch_over_one_at_a_time"], "target_ratio": 3.0,
            "launch": "one packed box table (all replicas) per kernel launch, each 100-step call a captured CUDA "
                      "graph; not a persistent kernel: persistent grids of 2-8 blocks per SM measured slower "
                      "(+10 % to +190 %) than one tile per block on this engine",
            "gpu_launches": r["gpu_launches"], "status_bits": r["status_bits"]}


def time_slice_profile(engine_mod, system, nslices: int, shape, dev, torch, steps: int = 20):
    """Cost of the slice stress profile (CMonitor::AddBeadStress & co.) on a
    sample step: per-kernel CUDA events over ``steps`` steps that all sample,
    with and without the profile, mixed precision."""
    from osprey_dpd_b200 import autotune
    out = {"slices": nslices}
    for on in (False, True):
        eng = engine_mod.DpdEngine.from_system(system, precision=engine_mod.MIXED, device=dev.index)
        if shape:
            autotune.apply_shape(eng, shape)
        if on:
            eng.set_slice_stress_for(system, nslices)
        eng.set_sample_period(1)
        eng.step(1, 3)
        eng.status()
        eng.profile(True)
        eng.step(4, steps)
        eng.status()
        p = eng.profile_read()
        per = {k: v["ms"] / v["launches"] for k, v in p.items() if v["launches"]}
        key = "with" if on else "without"
        out[f"sample_step_ms_{key}"] = sum(p[k]["ms"] for k in p) / steps
        if on:
            out["slice_pairs_ms"] = per.get("slices")
            out["bonds_ms_with"] = per.get("bonds")
            out["status"] = eng.status()
        else:
            out["bonds_ms_without"] = per.get("bonds")
        eng.close()
    out["timing"] = ("CUDA events around every kernel, kernels launched one by one, every step a sample step; "
                     "the profile is built on sample steps only")
    return out


def time_monitor(engine_mod, system, dev, reps: int = 10):
    """Wall time of one synchronous dpd_engine_monitor call (CMonitor sample
    data on the device) and of the full state download a host-side monitor
    would need instead, mixed precision, after 20 steps."""
    eng = engine_mod.DpdEngine.from_system(system, precision=engine_mod.MIXED, device=dev.index)
    eng.set_monitor_for(system)
    eng.step(1, 20)
    eng.status()
    eng.monitor()
    eng.download()
    t0 = time.perf_counter()
    for _ in range(reps):
        eng.monitor()
    t1 = time.perf_counter()
    for _ in range(reps):
        eng.download()
    t2 = time.perf_counter()
    eng.close()
    return {"monitor_ms": 1000.0 * (t1 - t0) / reps, "download_ms": 1000.0 * (t2 - t1) / reps,
            "timing": "host wall clock around synchronous calls"}


def read_traffic(n_beads: int, scheme: str = "full", workload: str = None):
    """Per-launch DRAM bytes of the pair kernel (full, half or staged) from the
    committed ncu summaries: the capture of this scheme on this workload when
    there is one, else the scheme's melt capture scaled to the bead count."""
    p = os.path.join(ROOT, "profiles", "pair_forces_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        table = json.load(fh)
    d = table.get(f"{scheme}_{workload}") or table.get(scheme) or {}
    if d.get("n_beads") == n_beads:
        return d["dram_bytes_read"] + d["dram_bytes_write"]
    per_bead = d.get("dram_bytes_per_bead")
    return None if per_bead is None else per_bead * n_beads


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload", default="bilayer", choices=["bilayer", "water", "binary", "polymer", "replicas"])
    ap.add_argument("--replicas", type=int, default=512)
    ap.add_argument("--graph-steps", type=int, default=100, help="steps per captured graph (replicas)")
    ap.add_argument("--e2e-reps", type=int, default=3)
    ap.add_argument("--cpu-steps", type=int, default=12, help="steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="default pair-kernel launch shape")
    ap.add_argument("--reproducible", action="store_true",
                    help="tune over the full-shell (bitwise reproducible) pair scheme only")
    ap.add_argument("--pair-scheme", choices=["auto", "full", "half", "staged"], default="auto",
                    help="fixed pair scheme with its default shape instead of the autotuner's choice")
    ap.add_argument("--precision", choices=["both", "mixed", "fp64"], default="both")
    ap.add_argument("--monitor", action="store_true",
                    help="also time dpd_engine_monitor against the state download it replaces")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the 6.3M-bead melt and the 512-replica sweep keys of the default line")
    ap.add_argument("--slices", type=int, default=0,
                    help="also time the slice stress profile over this many z slices on sample steps")
    ap.add_argument("--slab-exchange", type=int, default=0,
                    help="time the device slab engine instead: the workload split into this many z-slabs held "
                         "by this process on its one GPU (steps and exchanges, wall clock per phase)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")

    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    from osprey_dpd_b200 import ranks as R
    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    group = R.open_ranks("nccl", dev)
    from osprey_dpd_b200 import engine as E

    if args.slab_exchange:
        line = run_slab_exchange(args, dev, torch)
        if rank == 0:
            print(json.dumps(line), flush=True)
        group.close()
        return 0
    if args.workload == "replicas":
        line = run_replica_sweep(args, dev, torch, __import__("osprey_dpd_b200.engine", fromlist=["x"]))
        if rank == 0:
            print(json.dumps(line), flush=True)
        group.close()
        return 0
    system, desc = workload(args.workload, seed_offset=R.replica_seed_offset(rank))
    peaks, peak_kind = load_peaks()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    barrier = group.barrier
    max_over_ranks = group.max

    results = {}
    clocks = None
    precs = [("mixed", E.MIXED), ("fp64", E.FP64)]
    if args.precision != "both":
        precs = [p for p in precs if p[0] == args.precision]
    for prec_name, prec in precs:
        barrier()
        sampler = ClockSampler(local) if prec_name == "mixed" else None
        if sampler:
            sampler.start()
        tuned = tuned_shape(E, system, prec, dev, torch, not args.no_autotune, args.reproducible,
                            args.pair_scheme)
        torch.cuda.synchronize(dev)
        ms, prof, launches, status = time_engine(E, system, prec, args.steps, args.warmup, dev, torch, True,
                                                 tuned["shape"] if tuned else None)
        torch.cuda.synchronize(dev)
        barrier()
        if sampler:
            clocks = sampler.stop()
        total_ms = max_over_ranks(sum(ms))
        results[prec_name] = {"ms": ms, "total_ms": total_ms, "prof": prof, "launches": launches,
                              "status": status, "shape": tuned["shape"] if tuned else None,
                              "value": R.aggregate_rate(ws, system.n, args.steps, total_ms)}

    e2e_value = h2d_step = d2h_step = None
    e2e_times = []
    if not args.no_e2e:
        mshape = (results.get("mixed") or {}).get("shape")
        e2e_times, h2d_step, d2h_step = e2e_run(E, system, E.MIXED, args.e2e_reps, dev, torch, mshape)
        e2e_t = max_over_ranks(sum(e2e_times))
        e2e_value = R.aggregate_rate(ws, system.n, E2E_PERIOD * len(e2e_times), 1000.0 * e2e_t)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_reference_sample(system, args.cpu_steps)
            cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {exc}"}

    if rank != 0:
        group.close()
        return 0

    mixed = results.get("mixed") or results["fp64"]
    scheme = scheme_of(mixed["shape"])
    pair = mixed["prof"]["pair_forces"]
    t_pair = pair["ms"] / max(pair["launches"], 1) / 1000.0
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    issue_peak = sms * 128 * sm_max * 1e6
    achieved = SLOTS_PER_BEAD_STEP * system.n / t_pair
    kern_share = {k: round(v["ms"] / max(sum(x["ms"] for x in mixed["prof"].values()), 1e-12), 4)
                  for k, v in mixed["prof"].items() if v["launches"]}
    step_s = mixed["total_ms"] / 1000.0 / args.steps
    hbm_ach = ALG_BYTES_PER_BEAD_STEP["mixed"] * system.n / step_s
    line = {
        "metric": METRIC, "value": mixed["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mixed["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 forces / f64 state",
        "data": "synthetic (seeded generator, reference workload shapes)",
        "config": {"workload": desc, "n_beads": system.n, "cells": list(system.cells), "dt": system.dt,
                   "precision": "mixed", "l2": "flushed before every timed step (256 MiB write, then 256 MiB read so no dirty lines remain)",
                   "sample_period": SAMPLE_PERIOD, "pair_scheme": pair_scheme_name(mixed["shape"]),
                   "parallelism": "replicas" if ws > 1 else "single GPU"},
        "fp64": ({"value": results["fp64"]["value"], "ms_per_step": results["fp64"]["total_ms"] / args.steps,
                  "mixed_over_fp64": mixed["value"] / results["fp64"]["value"]} if "fp64" in results else None),
        "roofline": {"bound": "issue", "kernel": PAIR_KERNELS[scheme] + " (mixed)",
                     "achieved": achieved / 1e9, "peak": issue_peak / 1e9, "unit": "Gslot/s",
                     "frac": achieved / issue_peak,
                     "peak_basis": f"{sms} SMs x 128 FP32/INT32 lanes x {sm_max:.0f} MHz ({peak_kind} sm_max_mhz)",
                     "work_per_bead_step": SLOTS_PER_BEAD_STEP,
                     "avg_launch_ms": t_pair * 1000.0,
                     "timing": "CUDA events around every kernel on the engine's stream, in a 20-step pass "
                               "after the timed region (same engine and workload, kernels launched one by one)",
                     "traffic": read_traffic(system.n, scheme, args.workload)},
        "roofline_step_hbm": {"bound": "hbm", "achieved": hbm_ach / 1e9, "peak": float(peaks["hbm_gbs"]),
                              "unit": "GB/s", "frac": hbm_ach / 1e9 / float(peaks["hbm_gbs"]),
                              "bytes_per_bead_step": ALG_BYTES_PER_BEAD_STEP["mixed"], "basis": peak_kind},
        "kernel_share": kern_share,
        "launch_shape": {k: v["shape"] for k, v in results.items()},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_step, "d2h_bytes_per_step": d2h_step,
                "call": f"upload_beads + upload_topology + step({E2E_PERIOD}) + observables + download, host pinned "
                        f"buffers", "reps": len(e2e_times)},
        "gpu_launches": mixed["launches"],
        "clocks": clocks,
        "status_bits": {k: v["status"] for k, v in results.items()},
    }
    # the same fraction against the SM clock seen during the timed region,
    # when it sat below the maximum
    sm_seen = (clocks or {}).get("sm_mhz")
    if sm_seen:
        line["roofline"]["frac_at_observed_clock"] = achieved / (sms * 128 * float(sm_seen) * 1e6)
        line["roofline"]["observed_sm_mhz"] = float(sm_seen)
    if not args.no_extra and args.workload == "bilayer" and ws == 1:
        line["melt"] = time_melt(E, dev, torch, args.warmup)
        line["replica_sweep"] = time_sweep(E, dev, torch)
    if args.slices > 0:
        line["slice_profile"] = time_slice_profile(E, system, args.slices, mixed["shape"], dev, torch)
    if args.monitor:
        line["monitor"] = time_monitor(E, system, dev)
    print(json.dumps(line), flush=True)
    group.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
