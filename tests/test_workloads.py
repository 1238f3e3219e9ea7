"""Synthetic workloads: sizes of the five benchmark systems, the reference's
polymer-count arithmetic, wrapped vs unwrapped positions."""
import math

import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W


def test_benchmark_system_sizes():
    assert W.water(10).n == 3000
    b = W.binary_mixture(32)
    assert b.n == 98304 and int((b.types == 0).sum()) == 49152
    bl = W.bilayer()
    assert bl.n == 393216 and len(bl.bond_head) == 48000 and len(bl.angle_first) == 24000
    assert int((bl.types == 2).sum()) == 339216


def test_polymer_solution_size_small():
    s = W.polymer_solution(cells=(16, 16, 16))
    n = 3 * 16 ** 3
    chains = math.floor(0.3 * n / 16)
    assert s.n == n and len(s.bond_head) == chains * 15


@pytest.mark.parametrize("make", [lambda: W.bilayer(), lambda: W.polymer_solution(cells=(20, 20, 20)),
                                  lambda: W.water(7)])
def test_reference_polymer_counts_are_reproduced(make):
    s = make()
    fr = W.polymer_fractions(s)
    L = s.box
    total = s.density * L[0] * L[1] * L[2]
    nal = 0.0
    for p, f in zip(s.polymers, fr):
        nal += float(len(p.beads)) * f
    assert [int(f * total / nal) for f in fr] == [p.count for p in s.polymers]
    assert sum(fr) <= 1.00000001


def test_positions_wrapped_and_unwrapped_consistent():
    s = W.polymer_solution(cells=(12, 12, 12))
    L = s.box
    assert np.all(s.x >= 0) and np.all(s.x < L)
    k = (s.unpbc - s.x) / L
    assert np.allclose(k, np.round(k), atol=1e-12)


def test_replica_table():
    edges, fracs, a_ab, seeds = W.replica_table(512)
    assert edges.min() >= 8 and edges.max() <= 24
    assert 0.1 <= fracs.min() and fracs.max() <= 0.5
    assert a_ab[0] == 25.0 and abs(a_ab[-1] - 60.0) < 1e-12
    assert len(set(seeds.tolist())) == 512
