"""Seeded synthetic DPD systems and their Osprey-DPD input files.

The benchmark systems are the five named workloads of this engine: a water box,
a binary A/B mixture, an H3T6 lipid bilayer in water, a melt of 16-bead chains
in solvent and a batch of A/B replicas.  No public data set is involved; each
system is generated from a fixed seed with the shapes, sizes and value
distributions of those workloads.

A system is described the way Osprey-DPD describes it:

* bead types with the conservative ``a_ij`` and dissipative ``gamma_ij`` tables
  (``Bead`` blocks, InputDPDFile.cpp:466-520);
* beads numbered 1..N in polymer order, polymer types in declaration order and
  beads in shape order (InitialState.cpp:451-505);
* Hookean bonds (head id, tail id, k2, l0) and bond pairs (first bond, second
  bond, k3, phi0 in radians) with the reference's head/tail convention: in a
  linear shape the bond between consecutive beads p_k, p_k+1 has head p_k+1 and
  tail p_k, and a bond pair joins bond k (first) and bond k+1 (second);
* positions wrapped into [0, L), unwrapped positions (``unPBC``), velocities
  and forces (zero, as after the reference's random and lamella builders).

``write_dmpci`` writes an input file whose polymer fractions make the
reference build exactly the same numbers of polymers
(CInitialState::CreatePolymers truncates, InitialState.cpp:466-474), so the
reference and this engine can run the same system once the state is injected.
"""
from __future__ import annotations

import dataclasses
import math
import struct
from typing import List, Sequence, Tuple

import numpy as np

BASE_SEED = 20261203


@dataclasses.dataclass
class PolymerSpec:
    name: str
    beads: Tuple[str, ...]      # linear shape, bead type names in order
    count: int


@dataclasses.dataclass
class BondSpec:
    name1: str
    name2: str
    k2: float
    l0: float


@dataclasses.dataclass
class BondPairSpec:
    name1: str
    name2: str
    name3: str
    k3: float
    phi0_deg: float


@dataclasses.dataclass
class DpdSystem:
    """A complete DPD system: box, parameters, beads and topology."""

    name: str
    cells: Tuple[int, int, int]
    widths: Tuple[float, float, float]
    density: float
    dt: float
    lam: float
    kT: float
    seed: int
    type_names: List[str]
    a: np.ndarray               # (T, T) float64
    gamma: np.ndarray           # (T, T) float64
    polymers: List[PolymerSpec]
    bond_specs: List[BondSpec]
    bondpair_specs: List[BondPairSpec]
    ids: np.ndarray             # (N,) int64, 1..N
    types: np.ndarray           # (N,) int32
    movable: np.ndarray         # (N,) uint8
    x: np.ndarray               # (N, 3) float64, wrapped
    unpbc: np.ndarray           # (N, 3) float64, unwrapped
    v: np.ndarray               # (N, 3) float64
    f: np.ndarray               # (N, 3) float64
    bond_head: np.ndarray       # (nb,) int64 bead ids
    bond_tail: np.ndarray
    bond_k2: np.ndarray
    bond_l0: np.ndarray
    angle_first: np.ndarray     # (na,) int64 bond indices
    angle_second: np.ndarray
    angle_k3: np.ndarray
    angle_phi0: np.ndarray      # radians
    bond_type: np.ndarray = None    # (nb,) int32: index of the bond's Bond line (CBond::GetType)
    angle_type: np.ndarray = None   # (na,) int32: index of the pair's BondPair line (CBondPair::GetType)

    @property
    def n(self) -> int:
        return int(self.ids.shape[0])

    @property
    def box(self) -> np.ndarray:
        return np.array([c * w for c, w in zip(self.cells, self.widths)], dtype=np.float64)

    @property
    def ncells(self) -> int:
        return int(self.cells[0] * self.cells[1] * self.cells[2])

    def copy(self) -> "DpdSystem":
        return dataclasses.replace(
            self,
            **{f.name: (getattr(self, f.name).copy() if isinstance(getattr(self, f.name), np.ndarray)
                        else getattr(self, f.name))
               for f in dataclasses.fields(self)})


# --------------------------------------------------------------------- helpers

def _sym(T: int, entries: dict, names: Sequence[str]) -> np.ndarray:
    m = np.zeros((T, T), dtype=np.float64)
    for (p, q), val in entries.items():
        i, j = names.index(p), names.index(q)
        m[i, j] = m[j, i] = val
    return m


def maxwell_velocities(rng: np.random.Generator, n: int, kT: float) -> np.ndarray:
    """Gaussian velocities, zero net momentum, rescaled to sum(v^2)/3N = kT."""
    v = rng.standard_normal((n, 3))
    v -= v.mean(axis=0, keepdims=True)
    if kT > 0 and n > 1:
        v *= math.sqrt(kT * 3 * n / float(np.sum(v * v)))
    else:
        v[:] = 0.0
    return v


def _wrap(u: np.ndarray, L: np.ndarray) -> np.ndarray:
    x = u - np.floor(u / L) * L
    # floor can round a value just below L up to L; keep x in [0, L)
    x = np.where(x >= L, x - L, x)
    return np.where(x < 0, x + L, x)


def _linear_topology(polymers: Sequence[PolymerSpec], bond_specs: Sequence[BondSpec],
                     bp_specs: Sequence[BondPairSpec], names: Sequence[str]):
    """Bonds and bond pairs of linear polymers in the reference's order and
    head/tail convention (checked against the reference's own topology)."""
    bk = {}
    for q, b in enumerate(bond_specs):
        bk[(b.name1, b.name2)] = bk[(b.name2, b.name1)] = (b.k2, b.l0, q)
    pk = {}
    for q, p in enumerate(bp_specs):
        pk[(p.name1, p.name2, p.name3)] = pk[(p.name3, p.name2, p.name1)] = (p.k3, math.radians(p.phi0_deg), q)
    hs, ts, ks, ls, fs, ss, k3l, phl, bts, ats = [], [], [], [], [], [], [], [], [], []
    next_id = 1
    bond_base = 0
    for poly in polymers:
        m = len(poly.beads)
        tb = []                      # (head offset, tail offset, k2, l0) per template bond
        for k in range(m - 1):
            key = (poly.beads[k], poly.beads[k + 1])
            if key not in bk:
                raise ValueError(f"no Bond type for {key}")
            tb.append((k, k + 1) + bk[key])
        ta = []                      # (first bond, second bond, k3, phi0) per template pair
        for k in range(m - 2):
            key = (poly.beads[k], poly.beads[k + 1], poly.beads[k + 2])
            if key in pk:
                ta.append((k + 1, k) + pk[key])
        if poly.count and tb:
            c = poly.count
            nbp = len(tb)
            start = (np.arange(c, dtype=np.int64) * m + next_id)[:, None]
            hs.append((start + np.array([b[0] for b in tb])[None, :]).ravel())
            ts.append((start + np.array([b[1] for b in tb])[None, :]).ravel())
            ks.append(np.tile(np.array([b[2] for b in tb]), c))
            ls.append(np.tile(np.array([b[3] for b in tb]), c))
            bts.append(np.tile(np.array([b[4] for b in tb]), c))
            if ta:
                bstart = (bond_base + np.arange(c, dtype=np.int64) * nbp)[:, None]
                fs.append((bstart + np.array([a[0] for a in ta])[None, :]).ravel())
                ss.append((bstart + np.array([a[1] for a in ta])[None, :]).ravel())
                k3l.append(np.tile(np.array([a[2] for a in ta]), c))
                phl.append(np.tile(np.array([a[3] for a in ta]), c))
                ats.append(np.tile(np.array([a[4] for a in ta]), c))
            bond_base += c * nbp
        next_id += poly.count * m
    cat = lambda xs, dt: (np.concatenate(xs).astype(dt) if xs else np.zeros(0, dtype=dt))
    return (cat(hs, np.int64), cat(ts, np.int64), cat(ks, np.float64), cat(ls, np.float64),
            cat(fs, np.int64), cat(ss, np.int64), cat(k3l, np.float64), cat(phl, np.float64),
            cat(bts, np.int32), cat(ats, np.int32))


def _assemble(name, cells, widths, density, dt, lam, kT, seed, type_names, a, gamma,
              polymers, bond_specs, bp_specs, types, unpbc, v) -> DpdSystem:
    n = types.shape[0]
    L = np.array([c * w for c, w in zip(cells, widths)], dtype=np.float64)
    x = _wrap(unpbc, L)
    hb, tb, k2, l0, fa, sa, k3, phi, bty, aty = _linear_topology(polymers, bond_specs, bp_specs, type_names)
    return DpdSystem(
        name=name, cells=tuple(cells), widths=tuple(float(w) for w in widths), density=density,
        dt=dt, lam=lam, kT=kT, seed=seed, type_names=list(type_names), a=a, gamma=gamma,
        polymers=list(polymers), bond_specs=list(bond_specs), bondpair_specs=list(bp_specs),
        ids=np.arange(1, n + 1, dtype=np.int64), types=types.astype(np.int32),
        movable=np.ones(n, dtype=np.uint8), x=x, unpbc=unpbc.astype(np.float64),
        v=v.astype(np.float64), f=np.zeros((n, 3), dtype=np.float64),
        bond_head=hb, bond_tail=tb, bond_k2=k2, bond_l0=l0,
        angle_first=fa, angle_second=sa, angle_k3=k3, angle_phi0=phi, bond_type=bty, angle_type=aty)


# ------------------------------------------------------------------ workloads

def water(n: int = 10, density: float = 3.0, seed: int = BASE_SEED + 1, dt: float = 0.02,
          kT: float = 1.0, a: float = 25.0, gamma: float = 4.5) -> DpdSystem:
    """Single-component DPD water in an n^3 periodic box of unit cells."""
    rng = np.random.default_rng(seed)
    N = int(round(density * n ** 3))
    L = np.full(3, float(n))
    u = rng.random((N, 3)) * L
    v = maxwell_velocities(rng, N, kT)
    names = ["W"]
    return _assemble("water", (n, n, n), (1.0, 1.0, 1.0), density, dt, 0.5, kT, seed, names,
                     np.array([[a]]), np.array([[gamma]]), [PolymerSpec("Water", ("W",), N)], [], [],
                     np.zeros(N, dtype=np.int32), u, v)


def binary_mixture(n: int = 32, density: float = 3.0, seed: int = BASE_SEED + 2, a_ab: float = 50.0,
                   frac_a: float = 0.5, dt: float = 0.02, kT: float = 1.0, gamma: float = 4.5,
                   cells: Tuple[int, int, int] = None) -> DpdSystem:
    """Binary A/B mixture, randomly mixed: ids 1..N_A are A, the rest B."""
    cells = cells or (n, n, n)
    rng = np.random.default_rng(seed)
    V = cells[0] * cells[1] * cells[2]
    N = int(round(density * V))
    na = int(round(frac_a * N))
    L = np.array(cells, dtype=np.float64)
    u = rng.random((N, 3)) * L
    v = maxwell_velocities(rng, N, kT)
    names = ["A", "B"]
    am = _sym(2, {("A", "A"): 25.0, ("B", "B"): 25.0, ("A", "B"): a_ab}, names)
    gm = np.full((2, 2), gamma)
    types = np.concatenate([np.zeros(na, np.int32), np.ones(N - na, np.int32)])
    return _assemble("binary", cells, (1.0, 1.0, 1.0), density, dt, 0.5, kT, seed, names, am, gm,
                     [PolymerSpec("A", ("A",), na), PolymerSpec("B", ("B",), N - na)], [], [],
                     types, u, v)


def bilayer(cells: Tuple[int, int, int] = (64, 64, 32), nlipids: int = 6000, density: float = 3.0,
            seed: int = BASE_SEED + 3, dt: float = 0.02, kT: float = 1.0, gamma: float = 4.5,
            k3: float = 20.0, with_htt: bool = False, phi0_deg: float = 0.0) -> DpdSystem:
    """H3T6 lipids in two leaflets about the box mid-plane (heads outward),
    chains along z with 0.5 spacing on a jittered lateral lattice; water fills
    the box outside the bilayer slab.  Lipids are declared first (ids 1..9*nlipids)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = cells
    V = nx * ny * nz
    N = int(round(density * V))
    shape = ("H", "H", "H", "T", "T", "T", "T", "T", "T")
    m = len(shape)
    nw = N - nlipids * m
    if nw < 0:
        raise ValueError("too many lipids for the box")
    zmid = 0.5 * nz
    per = [nlipids - nlipids // 2, nlipids // 2]           # upper, lower leaflet
    lat = []
    for cnt in per:
        g = int(math.ceil(math.sqrt(cnt * nx / ny)))
        h = int(math.ceil(cnt / g))
        gx, gy = np.meshgrid((np.arange(g) + 0.5) * nx / g, (np.arange(h) + 0.5) * ny / h, indexing="ij")
        pts = np.stack([gx.ravel(), gy.ravel()], axis=1)
        pick = rng.permutation(pts.shape[0])[:cnt]
        jit = (rng.random((cnt, 2)) - 0.5) * 0.5 * np.array([nx / g, ny / h])
        lat.append(pts[pick] + jit)
    chains = []
    for leaf, cnt in enumerate(per):
        sgn = 1.0 if leaf == 0 else -1.0
        # bead k of the chain: heads (k=0) outermost, last tail at the mid-plane
        zoff = sgn * (0.25 + 0.5 * (m - 1 - np.arange(m)))
        c = np.empty((cnt, m, 3))
        c[:, :, 0] = lat[leaf][:, 0:1]
        c[:, :, 1] = lat[leaf][:, 1:2]
        c[:, :, 2] = zmid + zoff[None, :]
        chains.append(c)
    lip = np.concatenate(chains, axis=0).reshape(-1, 3)
    slab_lo = zmid - 0.25 - 0.5 * (m - 1) - 0.25
    slab_hi = zmid + 0.25 + 0.5 * (m - 1) + 0.25
    wz_len = nz - (slab_hi - slab_lo)
    w = rng.random((nw, 3)) * np.array([nx, ny, wz_len])
    w[:, 2] = np.where(w[:, 2] < slab_lo, w[:, 2], w[:, 2] + (slab_hi - slab_lo))
    u = np.concatenate([lip, w], axis=0)
    v = maxwell_velocities(rng, N, kT)
    names = ["H", "T", "W"]
    am = _sym(3, {("H", "H"): 30.0, ("H", "T"): 35.0, ("T", "T"): 10.0, ("H", "W"): 30.0,
                  ("T", "W"): 75.0, ("W", "W"): 25.0}, names)
    gm = np.full((3, 3), gamma)
    tmap = {"H": 0, "T": 1, "W": 2}
    types = np.concatenate([np.tile(np.array([tmap[s] for s in shape], np.int32), nlipids),
                            np.full(nw, 2, np.int32)])
    bonds = [BondSpec("H", "H", 128.0, 0.5), BondSpec("H", "T", 128.0, 0.5), BondSpec("T", "T", 128.0, 0.5)]
    bps = [BondPairSpec("T", "T", "T", k3, phi0_deg)]
    if with_htt:
        bps.append(BondPairSpec("H", "T", "T", k3, phi0_deg))
    return _assemble("bilayer", cells, (1.0, 1.0, 1.0), density, dt, 0.5, kT, seed, names, am, gm,
                     [PolymerSpec("Lipid", shape, nlipids), PolymerSpec("Water", ("W",), nw)],
                     bonds, bps, types, u, v)


def polymer_solution(n: int = 128, density: float = 3.0, frac_polymer: float = 0.3, chain: int = 16,
                     seed: int = BASE_SEED + 4, dt: float = 0.02, kT: float = 1.0, gamma: float = 4.5,
                     cells: Tuple[int, int, int] = None) -> DpdSystem:
    """Linear P_chain chains as random walks of step 0.5 (unwrapped positions
    kept) in solvent S.  Chains are declared first."""
    cells = cells or (n, n, n)
    rng = np.random.default_rng(seed)
    V = cells[0] * cells[1] * cells[2]
    N = int(round(density * V))
    nchains = int(math.floor(frac_polymer * N / chain))
    ns = N - nchains * chain
    L = np.array(cells, dtype=np.float64)
    start = rng.random((nchains, 1, 3)) * L
    steps = rng.standard_normal((nchains, chain - 1, 3))
    steps *= 0.5 / np.linalg.norm(steps, axis=2, keepdims=True)
    walk = np.concatenate([start, start + np.cumsum(steps, axis=1)], axis=1).reshape(-1, 3)
    sol = rng.random((ns, 3)) * L
    u = np.concatenate([walk, sol], axis=0)
    v = maxwell_velocities(rng, N, kT)
    names = ["P", "S"]
    am = _sym(2, {("P", "P"): 25.0, ("S", "S"): 25.0, ("P", "S"): 35.0}, names)
    gm = np.full((2, 2), gamma)
    types = np.concatenate([np.zeros(nchains * chain, np.int32), np.ones(ns, np.int32)])
    return _assemble("polymer", cells, (1.0, 1.0, 1.0), density, dt, 0.5, kT, seed, names, am, gm,
                     [PolymerSpec("Chain", ("P",) * chain, nchains), PolymerSpec("Solvent", ("S",), ns)],
                     [BondSpec("P", "P", 128.0, 0.5)], [], types, u, v)


def replica_table(nrep: int = 512, seed: int = BASE_SEED + 1000, lo: int = 8, hi: int = 24):
    """Parameters of the batched A/B sweep: per replica edge L_r ~ U{lo..hi},
    A fraction f_r ~ U[0.1, 0.5], a_AB swept 25 -> 60, own seed."""
    rng = np.random.default_rng(seed)
    edges = rng.integers(lo, hi + 1, size=nrep)
    fracs = rng.uniform(0.1, 0.5, size=nrep)
    a_ab = 25.0 + 35.0 * np.arange(nrep) / max(nrep - 1, 1)
    seeds = seed + 1 + np.arange(nrep)
    return edges, fracs, a_ab, seeds


def replica(r: int, nrep: int = 512, seed: int = BASE_SEED + 1000) -> DpdSystem:
    edges, fracs, a_ab, seeds = replica_table(nrep, seed)
    e = int(edges[r])
    return binary_mixture(n=e, seed=int(seeds[r]), a_ab=float(a_ab[r]), frac_a=float(fracs[r]))


# ---------------------------------------------------------- reference files

def polymer_fractions(system: DpdSystem) -> List[float]:
    """Number fractions for which CInitialState::CreatePolymers
    (InitialState.cpp:457-474) yields exactly each polymer's count, found by
    repeating its double arithmetic and nudging by ulps."""
    counts = [p.count for p in system.polymers]
    sizes = [len(p.beads) for p in system.polymers]
    tot = float(sum(counts))
    L = system.box
    total_beads = system.density * L[0] * L[1] * L[2]
    fr = [c / tot for c in counts]

    def built(fr):
        s = 0.0
        for k in range(len(fr)):
            s += float(sizes[k]) * fr[k]
        return [int(fr[k] * total_beads / s) for k in range(len(fr))]

    for _ in range(200):
        got = built(fr)
        if got == counts:
            break
        for k in range(len(fr)):
            if got[k] < counts[k]:
                fr[k] = math.nextafter(fr[k], 2.0)
            elif got[k] > counts[k]:
                fr[k] = math.nextafter(fr[k], -1.0)
    if built(fr) != counts:
        raise ValueError("no polymer fractions reproduce the bead counts")
    if sum(fr) > 1.00000001:
        raise ValueError("polymer fractions exceed the reference's sum limit")
    return fr


def lamella_block(polymer: str, normal=(0, 0, 1), centre: float = 0.5, thickness: float = 5.0,
                  linearise: bool = True, upper_fraction: float = 0.5) -> List[str]:
    """The `State lamella` block of a control data file (CInitialStateLamella,
    InitialStateLamella.cpp): the bilayer polymer, the normal axis, the
    mid-plane as a fraction of the box length, the bilayer thickness, straight
    or scattered chains, the fraction in the upper monolayer; no polymerised
    bonds."""
    return ["State\tlamella", f"        Polymer\t\t\t{polymer}",
            f"        Normal\t\t\t{normal[0]} {normal[1]} {normal[2]}", f"        Centre\t\t\t{centre!r}",
            f"        Thickness\t\t{thickness!r}", f"        Linearise\t\t{1 if linearise else 0}",
            f"        UpperFraction\t{upper_fraction!r}", "        Polymerise\t\t0"]


def write_dmpci(system: DpdSystem, path: str, steps: int, kT: float = None, seed: int = None,
                gamma_scale: float = 1.0, title: str = "synthetic", grid_z: int = 1,
                state: List[str] = None) -> None:
    """Osprey-DPD control data file (InputDPDFile.cpp:400-800) for ``system``
    running ``steps`` steps with sampling, display and restart only at the end;
    ``grid_z`` analysis-grid slices along z (the slice stress profile's);
    ``state`` the initial-state block (default `State random`, or
    lamella_block(...))."""
    T = len(system.type_names)
    lines = ["dpd", "", f'Title\t" {title} "', "Date    03/12/26",
             f'Comment\t" generated {system.name} system "', ""] + (state or ["State\trandom"]) + [""]
    for i, name in enumerate(system.type_names):
        lines.append(f"Bead  {name}")
        lines.append("      0.5")
        lines.append("      " + "  ".join(repr(float(system.a[i, j])) for j in range(i + 1)))
        lines.append("      " + "  ".join(repr(float(system.gamma[i, j] * gamma_scale)) for j in range(i + 1)))
        lines.append("")
    for b in system.bond_specs:
        lines.append(f"Bond  {b.name1} {b.name2}  {b.k2!r}  {b.l0!r}")
    if system.bond_specs:
        lines.append("")
    for p in system.bondpair_specs:
        lines.append(f"BondPair  {p.name1} {p.name2} {p.name3}  {p.k3!r}  {p.phi0_deg!r}")
    if system.bondpair_specs:
        lines.append("")
    for p, fr in zip(system.polymers, polymer_fractions(system)):
        lines.append(f'Polymer  {p.name}  {fr!r}  " ({" ".join(p.beads)}) "')
    lines.append("")
    c, w = system.cells, system.widths
    lines += [f"Box   {c[0]} {c[1]} {c[2]}   {w[0]!r} {w[1]!r} {w[2]!r}",
              f"Density  {system.density!r}",
              f"Temp  {float(system.kT if kT is None else kT)!r}",
              f"RNGSeed  {-abs(int(system.seed if seed is None else seed)) % 2147483647}",
              f"Lambda  {system.lam!r}",
              f"Step  {system.dt!r}",
              f"Time  {steps}",
              f"SamplePeriod  {steps}",
              f"AnalysisPeriod  {steps}",
              f"DensityPeriod  {steps}",
              f"DisplayPeriod  {steps}",
              f"RestartPeriod  {steps}",
              f"Grid  1 1 {int(grid_z)}", ""]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_state(system: DpdSystem, path: str) -> None:
    """Bead state for the reference harness, records ordered by bead id."""
    n = system.n
    rec = np.zeros(n, dtype=[("id", "<i8"), ("type", "<i8"), ("x", "<f8", 3), ("u", "<f8", 3),
                             ("v", "<f8", 3), ("f", "<f8", 3)])
    rec["id"] = system.ids
    rec["type"] = system.types
    rec["x"] = system.x
    rec["u"] = system.unpbc
    rec["v"] = system.v
    rec["f"] = system.f
    with open(path, "wb") as fh:
        fh.write(b"DPDSTATE")
        fh.write(struct.pack("<q", n))
        fh.write(rec.tobytes())


def read_dump(path: str):
    """Reference harness dump: dict of id-ordered arrays."""
    with open(path, "rb") as fh:
        if fh.read(8) != b"DPDDUMP1":
            raise ValueError("not a DPDDUMP1 file")
        n, steps = struct.unpack("<qq", fh.read(16))
        dt = np.dtype([("id", "<i8"), ("type", "<i8"), ("x", "<f8", 3), ("u", "<f8", 3), ("v", "<f8", 3),
                       ("f", "<f8", 3), ("stress", "<f8", 9)])
        rec = np.frombuffer(fh.read(n * dt.itemsize), dtype=dt)
    return {"n": n, "steps": steps, "id": rec["id"].copy(), "type": rec["type"].copy(),
            "x": rec["x"].copy(), "unpbc": rec["u"].copy(), "v": rec["v"].copy(), "f": rec["f"].copy(),
            "stress": rec["stress"].copy()}


def read_slices(path: str):
    """Slice stress dump of the reference harness (--slices)."""
    with open(path, "rb") as fh:
        if fh.read(8) != b"DPDSLICE":
            raise ValueError("not a DPDSLICE file")
        S, T, nbt, nbpt, nb, na = struct.unpack("<6q", fh.read(48))
        rd = lambda cnt: np.frombuffer(fh.read(8 * cnt), dtype="<f8").copy()
        pair = rd(S * T * T * 9).reshape(S, T * T, 9)
        bond = rd(S * nbt * 9).reshape(S, nbt, 9)
        bp = rd(S * nbpt * 9).reshape(S, nbpt, 9)
        btype = np.frombuffer(fh.read(8 * nb), dtype="<i8").copy()
        atype = np.frombuffer(fh.read(8 * na), dtype="<i8").copy()
    return {"pair": pair, "bond": bond, "bondpair": bp, "bond_type": btype, "angle_type": atype}


def read_topology(path: str):
    with open(path, "rb") as fh:
        if fh.read(8) != b"DPDTOPO1":
            raise ValueError("not a DPDTOPO1 file")
        (nb,) = struct.unpack("<q", fh.read(8))
        bt = np.dtype([("h", "<i8"), ("t", "<i8"), ("k2", "<f8"), ("l0", "<f8")])
        b = np.frombuffer(fh.read(nb * bt.itemsize), dtype=bt)
        (na,) = struct.unpack("<q", fh.read(8))
        at = np.dtype([("f", "<i8"), ("s", "<i8"), ("k3", "<f8"), ("phi0", "<f8")])
        a = np.frombuffer(fh.read(na * at.itemsize), dtype=at)
    return {"bond_head": b["h"].copy(), "bond_tail": b["t"].copy(), "bond_k2": b["k2"].copy(),
            "bond_l0": b["l0"].copy(), "angle_first": a["f"].copy(), "angle_second": a["s"].copy(),
            "angle_k3": a["k3"].copy(), "angle_phi0": a["phi0"].copy()}
