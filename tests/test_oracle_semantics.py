"""Edge cases of the reference's step, checked on the CPU oracle (which is
pinned to the reference): frozen beads, the incremental cell move and its
audit, beads on cell faces, the box boundary, and the Philox pair stream."""
import numpy as np
import pytest

from osprey_dpd_b200 import workloads as W


def _philox2x32_10(c0, c1, k):
    M, Wc = 0xD256D193, 0x9E3779B9
    for _ in range(10):
        p = M * c0
        c0, c1 = ((p >> 32) ^ k ^ c1) & 0xFFFFFFFF, p & 0xFFFFFFFF
        k = (k + Wc) & 0xFFFFFFFF
    return c0


def _step_key(seed, step):
    s = (seed & 0xFFFFFFFF) ^ (((seed >> 32) * 0x85EBCA6B) & 0xFFFFFFFF)
    s ^= s >> 16
    s = (s * 0x7FEB352D) & 0xFFFFFFFF
    s ^= s >> 15
    return (s + step * 0xC2B2AE35) & 0xFFFFFFFF


def test_philox_stream_matches_the_written_algorithm(oracle_mod):
    rng = np.random.default_rng(1)
    for _ in range(200):
        seed = int(rng.integers(0, 2**63))
        step = int(rng.integers(0, 2**31))
        a, b = sorted(int(v) for v in rng.integers(1, 2**31, size=2))
        assert oracle_mod.philox_pair(seed, step, a, b) == _philox2x32_10(a, b, _step_key(seed, step))


def test_philox_uniform_statistics(oracle_mod):
    u = np.array([oracle_mod.philox_pair(20261203, 5, i, i + 7) for i in range(1, 20001)]) / 2.0**32
    assert abs(u.mean() - 0.5) < 0.01 and abs(u.var() - 1 / 12) < 0.003


def test_philox_noise_keeps_pair_forces_antisymmetric(oracle_mod):
    s = W.water(8)
    o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    o.step(1, 3)
    f = o.state()["f"]
    assert np.max(np.abs(f.sum(axis=0))) < 1e-9 * np.sqrt((f ** 2).sum())


def test_frozen_beads_do_not_move_and_keep_accumulating_force(oracle_mod):
    s = W.water(6)
    s.movable[:50] = 0
    o = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    o.step(1, 1)
    st1 = o.state()
    o.step(2, 1)
    st2 = o.state()
    assert np.array_equal(st2["x"][:50], s.x[:50]) and np.array_equal(st2["v"][:50], s.v[:50])
    assert not np.array_equal(st2["x"][50:], s.x[50:])
    # CCNTCell::UpdatePos skips non-movable beads, so their force is never reset
    # (CNTCell.cpp:1640-1760): step 2 adds to step 1's sum
    o2 = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    o2.step(2, 1)
    assert not np.allclose(st2["f"][:50], o2.state()["f"][:50])


def test_bead_on_the_upper_cell_face_stays_in_its_cell(oracle_mod):
    """x == TR is not 'x > TR': the reference keeps the bead in its old cell
    (CNTCell.cpp:1768) while floor(x/w) files it one cell up."""
    s = W.water(5, density=0.2)          # 25 beads, few interactions
    s.v[:] = 0.0
    s.f[:] = 0.0
    s.x[0] = [1.5, 1.5, 1.5]
    s.unpbc[0] = s.x[0]
    s.v[0] = [0.5 / s.dt, 0.0, 0.0]      # lands exactly on x = 2.0
    o = oracle_mod.Oracle(s, kT=0.0, gamma_scale=0.0)
    o.step(1, 1)
    cell = o.cells()[0]
    assert o.state()["x"][0, 0] == 2.0
    assert cell == 1 + 5 * (1 + 5 * 1)       # still ix = 1
    assert o.cell_errors() >= 1              # the audit formula disagrees


def test_two_cell_jump_is_misfiled_and_reported(oracle_mod):
    s = W.water(6, density=0.2)
    s.v[:] = 0.0
    s.f[:] = 0.0
    s.x[0] = [1.2, 1.5, 1.5]
    s.unpbc[0] = s.x[0]
    s.v[0] = [1.9 / s.dt, 0.0, 0.0]      # x: 1.2 -> 3.1, two cells along
    o = oracle_mod.Oracle(s, kT=0.0, gamma_scale=0.0)
    o.step(1, 1)
    assert o.cells()[0] == 2 + 6 * (1 + 6 * 1)   # only one cell further, as the reference files it
    assert o.cell_errors() == 1


def test_crossing_the_box_boundary_wraps_x_not_unpbc(oracle_mod):
    s = W.water(6, density=0.2)
    s.v[:] = 0.0
    s.f[:] = 0.0
    s.x[0] = [5.95, 3.5, 0.02]
    s.unpbc[0] = s.x[0]
    s.v[0] = [0.1 / s.dt, 0.0, -0.05 / s.dt]
    o = oracle_mod.Oracle(s, kT=0.0, gamma_scale=0.0)
    o.step(1, 1)
    st = o.state()
    assert np.allclose(st["x"][0], [0.05, 3.5, 5.97])
    assert np.allclose(st["unpbc"][0], [6.05, 3.5, -0.03])
    assert o.cells()[0] == 0 + 6 * (3 + 6 * 5)
