"""Parity with the CPU oracle at the sizes the benchmark runs.

The workloads of the throughput measurements, at full size:
  binary32  A/B mixture, 32^3 cells, 98,304 beads, a_AB = 50
  bilayer   H3T6 bilayer in water, 64x64x32 cells, 393,216 beads, 48,000
            bonds, 24,000 bond pairs (the headline workload)
  polymer   16-bead chains in solvent, 128^3 cells, 6,291,456 beads,
            1,769,460 bonds
The oracle (the reference's algorithm in C, pinned bit for bit to the
reference binary) runs each case once; the engine runs it in both
precisions and with every pair scheme the benchmark can choose.
Bounds, as in the small-box parity tests:
  * thermostat off (gamma = 0), one step: positions bit-identical, forces
    within 1e-5 (mixed) / 1e-11 (FP64) of the force RMS, cells identical;
  * five thermostatted steps (Philox pair noise on both sides): forces within
    1e-4 / 1e-10 of the force RMS, unPBC positions within 1e-6 / 1e-12;
    FP64 cells identical; mixed-precision cells identical except where a
    coordinate lies within 1e-6 of a cell face (the FP32 forces move x by
    ~1e-9, which can put such a bead on the other side of the face);
  * run to run, the half-shell schemes (atomics, so the FP32 summation order
    varies): two runs of the same five steps agree within the same bounds.
"""
import numpy as np
import pytest

from conftest import rel_err
from osprey_dpd_b200 import workloads as W

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

WORKLOADS = {
    "binary32": lambda: W.binary_mixture(32),
    "bilayer": lambda: W.bilayer(),
    "polymer": lambda: W.polymer_solution(),
}
# the pair schemes the benchmark's autotuner chooses from for a single box
SCHEMES = {"half": 1}


def _face_distance(x, widths):
    """Distance of every coordinate to its nearest CNT cell face."""
    w = np.asarray(widths)
    r = np.mod(x, w)
    return np.minimum(r, w - r)


def _engine(engine_mod, s, precision, scheme, **kw):
    eng = engine_mod.DpdEngine.from_system(s, precision=precision, device=0, **kw)
    eng.set_pair_scheme(scheme)
    return eng


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_full_size_one_step_without_thermostat(engine_mod, oracle_mod, name):
    s = WORKLOADS[name]()
    orc = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX, gamma_scale=0.0)
    orc.step(1, 1)
    o = orc.state()
    ocells = orc.cells()
    del orc
    for precision, tol in ((0, 1e-5), (1, 1e-11)):
        for sname, scheme in SCHEMES.items():
            eng = _engine(engine_mod, s, precision, scheme, gamma_scale=0.0)
            eng.step(1, 1)
            g = eng.download(stress=False)
            err = rel_err(g["f"], o["f"])
            print(f"\n{name} {sname} precision={precision}: force error {err:.2e} of RMS")
            assert np.array_equal(g["x"], o["x"]), "first-step drift must be bit-identical"
            assert err < tol
            assert np.array_equal(eng.cells(), ocells)
            assert eng.status() == 0
            eng.close()


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_full_size_five_thermostatted_steps(engine_mod, oracle_mod, name):
    s = WORKLOADS[name]()
    orc = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX)
    orc.step(1, 5)
    o = orc.state()
    ocells = orc.cells()
    del orc
    for precision, ftol, xtol in ((0, 1e-4, 1e-6), (1, 1e-10, 1e-12)):
        for sname, scheme in SCHEMES.items():
            eng = _engine(engine_mod, s, precision, scheme)
            eng.step(1, 5)
            g = eng.download(stress=False)
            ferr = rel_err(g["f"], o["f"])
            xerr = float(np.max(np.abs(g["unpbc"] - o["unpbc"])))
            print(f"\n{name} {sname} precision={precision}: force error {ferr:.2e} of RMS, unPBC {xerr:.2e}")
            assert ferr < ftol
            assert xerr < xtol
            cells = eng.cells()
            diff = np.nonzero(cells != ocells)[0]
            if precision == 1:
                assert diff.size == 0
            else:
                near = _face_distance(o["x"][diff], s.widths).min(axis=1) if diff.size else np.zeros(0)
                assert np.all(near < 1e-6), near
            assert eng.status() & ~engine_mod.STATUS_CELL_SKIP == 0
            eng.close()


@pytest.mark.parametrize("name", ["bilayer", "polymer"])
def test_half_shell_run_to_run_variation_is_bounded(engine_mod, name):
    """The half-shell schemes add partner forces with atomics, so the FP32 sum
    order changes between runs; two runs from the same state stay within the
    oracle bounds after five steps."""
    s = WORKLOADS[name]()
    for sname, scheme in SCHEMES.items():
        runs = []
        for _ in range(2):
            eng = _engine(engine_mod, s, 0, scheme)
            eng.step(1, 5)
            runs.append(eng.download(stress=False))
            eng.close()
        ferr = rel_err(runs[1]["f"], runs[0]["f"])
        xerr = float(np.max(np.abs(runs[1]["unpbc"] - runs[0]["unpbc"])))
        print(f"\n{name} {sname}: run-to-run force {ferr:.2e} of RMS, unPBC {xerr:.2e}")
        assert ferr < 1e-4
        assert xerr < 1e-6
