"""numpy restatement of the reference's CMonitor sample data, applied to a
state (positions, unPBC positions) -- the oracle for dpd_engine_monitor.

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the engine.

  CMonitor::CalculateSingleBeadData     Monitor.cpp:790-1040 (inertia, MSD)
  CMonitor::CalculateSinglePolymerData  Monitor.cpp:708-788
  CMonitor::CalculateSingleBondData     Monitor.cpp:1052-1174
  CMonitor::CalculateSingleBondPairData Monitor.cpp:1176-1273, with the
                                        observables of CBondPair::AddForce,
                                        BondPair.cpp:140-199
"""
from __future__ import annotations

import math

import numpy as np


def _min_image(d, L):
    # Monitor.cpp:733-752: one correction past half the box length
    d = d.copy()
    for k in range(3):
        hi = d[:, k] > 0.5 * L[k]
        lo = d[:, k] < -0.5 * L[k]
        d[hi, k] -= L[k]
        d[lo, k] += L[k]
    return d


def monitor(system, x, unpbc, initial_unpbc, step: int, dt: float):
    """x, unpbc: (N, 3) in bead (upload) order; polymers as laid out by the
    workloads (ids 1..N, each polymer's beads consecutive)."""
    N = x.shape[0]
    T = len(system.type_names)
    L = system.box
    out = {}
    I = np.zeros(9)
    I[0] = np.sum(x[:, 1] ** 2 + x[:, 2] ** 2)
    I[1] = np.sum(-x[:, 0] * x[:, 1])
    I[2] = np.sum(-x[:, 0] * x[:, 2])
    I[4] = np.sum(x[:, 0] ** 2 + x[:, 2] ** 2)
    I[5] = np.sum(-x[:, 1] * x[:, 2])
    I[8] = np.sum(x[:, 0] ** 2 + x[:, 1] ** 2)
    I /= N
    I[3], I[6], I[7] = I[1], I[2], I[5]
    out["inertia"] = I.reshape(3, 3)
    d2 = np.sum((unpbc - initial_unpbc) ** 2, axis=1)
    pre = 6.0 * dt * step
    msd = np.zeros(T)
    for t in range(T):
        sel = system.types == t
        if sel.any():
            msd[t] = d2[sel].sum() / ((pre if pre > 0 else 1.0) * sel.sum())
    out["msd"] = msd
    # bonds (minimum image of wrapped positions)
    h = system.bond_head - 1
    tl = system.bond_tail - 1
    nbt = len(system.bond_specs)
    if len(h):
        r = np.sqrt(np.sum(_min_image(x[h] - x[tl], L) ** 2, axis=1))
        out["bond_length"] = np.array([r[system.bond_type == k].mean() if np.any(system.bond_type == k) else 0.0
                                       for k in range(nbt)])
        out["mean_bond_length"] = r.mean()
        out["mean_sq_bond_length"] = np.mean(r * r)
    else:
        out["bond_length"] = np.zeros(nbt)
        out["mean_bond_length"] = out["mean_sq_bond_length"] = 0.0
    # polymers
    ee = []
    nxt = 0
    for p in system.polymers:
        m = len(p.beads)
        heads = nxt + m * np.arange(p.count)
        tails = heads + m - 1
        r = np.sqrt(np.sum(_min_image(x[heads] - x[tails], L) ** 2, axis=1)) if p.count else np.zeros(0)
        ee.append(r.mean() if p.count else 0.0)
        nxt += m * p.count
    out["end_to_end"] = np.array(ee)
    # bond pairs (unPBC bond vectors)
    nbpt = len(system.bondpair_specs)
    acc = np.zeros((nbpt, 5))
    cnt = np.zeros(nbpt)
    for k in range(len(system.angle_first)):
        b1i, b2i = system.angle_first[k], system.angle_second[k]
        b1 = unpbc[system.bond_head[b1i] - 1] - unpbc[system.bond_tail[b1i] - 1]
        b2 = unpbc[system.bond_head[b2i] - 1] - unpbc[system.bond_tail[b2i] - 1]
        l1, l2 = math.sqrt(b1 @ b1), math.sqrt(b2 @ b2)
        P2 = phid = 0.0
        phi0 = float(system.angle_phi0[k])
        if l1 * l2 > 0.0001:
            dot = float(b1 @ b2)
            cos2 = (dot / (l1 * l1)) * (dot / (l2 * l2))
            if abs(dot) > 0.000001:
                pre_ = math.sqrt(1.0 / cos2 - 1.0)
                P2 = (0.5 * (3.0 * cos2 * (math.cos(phi0) + math.sin(phi0) * pre_) - 1.0) if phi0 > 0.0
                      else 0.5 * (3.0 * cos2 - 1.0))
            else:
                P2 = -0.5
            phid = math.acos(cos2) - phi0
        t = system.angle_type[k]
        acc[t] += (P2, l1, l2, phid, phid * phid)
        cnt[t] += 1
    bp = np.zeros((nbpt, 6))
    for t in range(nbpt):
        if cnt[t]:
            bp[t, :5] = acc[t] / cnt[t]
            bp[t, 5] = bp[t, 4] / (bp[t, 3] ** 2) if bp[t, 3] > 0 else 0.0
    out["bondpair"] = bp
    return out
