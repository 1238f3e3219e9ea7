"""Edge cases of the CUDA engine through the C ABI, against the CPU oracle:
frozen beads, beads landing on a cell face, multi-cell jumps, the box
boundary, non-unit cell widths, ragged boxes, bond pairs with a preferred
angle, bead-order invariance, and the error and status paths."""
import numpy as np
import pytest

from conftest import rel_err
from osprey_dpd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _sparse_box(n=6):
    s = W.water(n, density=0.2)
    s.v[:] = 0.0
    s.f[:] = 0.0
    return s


def _both(engine_mod, oracle_mod, s, precision=1, **kw):
    eng = engine_mod.DpdEngine.from_system(s, precision=precision, **kw)
    orc = oracle_mod.Oracle(s, noise=oracle_mod.NOISE_PHILOX, **kw)
    return eng, orc


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_frozen_beads(engine_mod, oracle_mod, precision):
    s = W.water(8)
    s.movable[::7] = 0
    eng, orc = _both(engine_mod, oracle_mod, s, precision)
    eng.step(1, 4)
    orc.step(1, 4)
    g, o = eng.download(), orc.state()
    fz = s.movable == 0
    assert np.array_equal(g["x"][fz], s.x[fz]) and np.array_equal(g["v"][fz], s.v[fz])
    ftol = 1e-4 if precision == 0 else 1e-10
    assert rel_err(g["f"], o["f"]) < ftol
    assert np.array_equal(eng.cells(), orc.cells())


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_frozen_beads_across_calls(engine_mod, oracle_mod, precision):
    """Frozen beads, bonded ones among them, over several calls: the last
    step of a call drifts the next step's state into separate buffers, which
    must carry the frozen beads' unchanged positions, images and cells too."""
    s = W.bilayer(cells=(12, 12, 12), nlipids=60)
    s.movable[::5] = 0
    eng, orc = _both(engine_mod, oracle_mod, s, precision)
    for first in (1, 3, 4):
        eng.step(first, 2 if first == 1 else 1)
    eng.step(5, 2)
    orc.step(1, 6)
    g, o = eng.download(), orc.state()
    fz = s.movable == 0
    assert np.array_equal(g["x"][fz], s.x[fz]) and np.array_equal(g["v"][fz], s.v[fz])
    assert np.array_equal(eng.cells(), orc.cells())
    assert rel_err(g["f"], o["f"]) < (1e-4 if precision == 0 else 1e-10)
    assert eng.status() == 0


def test_face_landing_bead_keeps_its_cell(engine_mod, oracle_mod):
    s = _sparse_box(5)
    s.x[0] = [1.5, 1.5, 1.5]
    s.unpbc[0] = s.x[0]
    s.v[0] = [0.5 / s.dt, 0.0, 0.0]
    eng, orc = _both(engine_mod, oracle_mod, s, kT=0.0, gamma_scale=0.0)
    eng.step(1, 1)
    orc.step(1, 1)
    assert eng.download()["x"][0, 0] == 2.0
    assert np.array_equal(eng.cells(), orc.cells())
    assert eng.status() & engine_mod.STATUS_CELL_SKIP   # the audit disagrees, as in the reference


def test_two_cell_jump_filed_like_the_reference(engine_mod, oracle_mod):
    s = _sparse_box(6)
    s.x[0] = [1.2, 1.5, 1.5]
    s.unpbc[0] = s.x[0]
    s.v[0] = [1.9 / s.dt, 0.0, 0.0]
    eng, orc = _both(engine_mod, oracle_mod, s, kT=0.0, gamma_scale=0.0)
    eng.step(1, 1)
    orc.step(1, 1)
    assert np.array_equal(eng.cells(), orc.cells())
    assert eng.status() == engine_mod.STATUS_CELL_SKIP and orc.cell_errors() == 1


def test_box_boundary_crossing(engine_mod, oracle_mod):
    s = _sparse_box(6)
    s.x[0] = [5.95, 3.5, 0.02]
    s.unpbc[0] = s.x[0]
    s.v[0] = [0.1 / s.dt, 0.0, -0.05 / s.dt]
    s.x[1] = [0.01, 5.99, 5.99]
    s.unpbc[1] = s.x[1] + np.array([-6.0, 12.0, 0.0])    # unPBC two images away
    s.v[1] = [-0.03 / s.dt, 0.02 / s.dt, 0.02 / s.dt]
    eng, orc = _both(engine_mod, oracle_mod, s, kT=0.0, gamma_scale=0.0)
    eng.step(1, 3)
    orc.step(1, 3)
    g, o = eng.download(), orc.state()
    assert np.array_equal(eng.cells(), orc.cells())
    assert np.allclose(g["x"], o["x"], rtol=0, atol=1e-12)
    assert np.allclose(g["unpbc"], o["unpbc"], rtol=0, atol=1e-12)


def _system_with_widths(widths=(1.5, 1.0, 1.25), cells=(5, 7, 6)):
    rng = np.random.default_rng(3)
    L = np.array(cells) * np.array(widths)
    N = int(3 * np.prod(L))
    u = rng.random((N, 3)) * L
    v = W.maxwell_velocities(rng, N, 1.0)
    names = ["A", "B"]
    a = np.array([[25.0, 40.0], [40.0, 25.0]])
    g = np.full((2, 2), 4.5)
    types = (np.arange(N) % 2).astype(np.int32)
    na = int((types == 0).sum())
    order = np.argsort(types, kind="stable")
    return W._assemble("widths", cells, widths, 3.0, 0.02, 0.5, 1.0, 77, names, a, g,
                       [W.PolymerSpec("A", ("A",), na), W.PolymerSpec("B", ("B",), N - na)], [], [],
                       types[order], u[order], v[order])


@pytest.mark.parametrize("scheme", [0, 1, 2], ids=["full", "half", "staged"])
@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_non_unit_cell_widths_and_ragged_box(engine_mod, oracle_mod, precision, scheme):
    s = _system_with_widths()
    eng, orc = _both(engine_mod, oracle_mod, s, precision)
    eng.set_pair_scheme(scheme)
    eng.step(1, 5)
    orc.step(1, 5)
    g, o = eng.download(), orc.state()
    ftol = 1e-4 if precision == 0 else 1e-10
    assert rel_err(g["f"], o["f"]) < ftol
    assert np.array_equal(eng.cells(), orc.cells())


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_bond_pairs_with_preferred_angle(engine_mod, oracle_mod, precision):
    s = W.bilayer(cells=(8, 8, 8), nlipids=16, with_htt=True, phi0_deg=30.0, seed=11)
    eng, orc = _both(engine_mod, oracle_mod, s, precision, gamma_scale=0.0)
    eng.step(1, 1)
    orc.step(1, 1)
    ftol = 1e-5 if precision == 0 else 1e-11
    assert rel_err(eng.download()["f"], orc.state()["f"]) < ftol


def test_bead_upload_order_does_not_change_forces(engine_mod):
    s = W.binary_mixture(cells=(7, 8, 9))
    e1 = engine_mod.DpdEngine.from_system(s, precision=1)
    e1.step(1, 2)
    f1 = e1.download()["f"]
    perm = np.random.default_rng(5).permutation(s.n)
    s2 = s.copy()
    for k in ("ids", "types", "movable", "x", "unpbc", "v", "f"):
        setattr(s2, k, getattr(s, k)[perm])
    e2 = engine_mod.DpdEngine.from_system(s2, precision=1, topology=False)
    e2.step(1, 2)
    f2 = np.empty_like(f1)
    f2[perm] = e2.download()["f"]
    assert rel_err(f2, f1) < 1e-11


def test_errors_and_status_words(engine_mod):
    s = W.water(6)
    eng = engine_mod.DpdEngine(s.cells, s.widths, s.dt, s.lam, s.kT, s.a, s.gamma, 1)
    with pytest.raises(engine_mod.EngineError, match="no beads"):
        eng.step(1, 1)
    bad = s.x.copy()
    bad[3] = [6.5, 1.0, 1.0]
    with pytest.raises(engine_mod.EngineError, match="outside the box"):
        eng.upload_beads(s.ids, s.types, s.movable, bad, None, s.v)
    eng.upload_beads(s.ids, s.types, s.movable, s.x, s.unpbc, s.v)
    v = s.v.copy()
    v[10] = [np.nan, 0.0, 0.0]
    with pytest.raises(engine_mod.EngineError, match="non-finite"):
        eng.upload_beads(s.ids, s.types, s.movable, s.x, s.unpbc, v)
    # a huge force yields a non-finite state that the status word reports
    f = np.zeros_like(s.x)
    f[10] = [1e308, 0.0, 0.0]
    eng.upload_beads(s.ids, s.types, s.movable, s.x, s.unpbc, s.v, f)
    eng.step(1, 1)
    assert eng.status() & engine_mod.STATUS_NONFINITE
    eng.close()


def test_parameter_mutators_follow_the_reference(engine_mod, oracle_mod):
    """ChangeTimeStepConstants, SetDPDBeadConsInt/DissInt and
    ToggleDPDBeadThermostat between steps (CNTCell.cpp:318-456)."""
    s = W.binary_mixture(cells=(6, 7, 8))
    eng, orc = _both(engine_mod, oracle_mod, s, 1)
    eng.step(1, 2)
    orc.step(1, 2)
    eng.set_dt(0.01)
    orc.set_dt(0.01)
    a = s.a.copy()
    g = s.gamma.copy()
    a[0, 1] = a[1, 0] = 60.0
    g[0, 1] = g[1, 0] = 2.0
    eng.set_pair_params(a, g)
    orc.set_pair(0, 1, 60.0, 2.0)
    eng.step(3, 2)
    orc.step(3, 2)
    assert rel_err(eng.download()["f"], orc.state()["f"]) < 1e-10
    # thermostat off zeroes gamma (dissipative and random forces) until restored
    eng.set_thermostat(False)
    orc.set_pair(0, 0, s.a[0, 0], 0.0)
    orc.set_pair(1, 1, s.a[1, 1], 0.0)
    orc.set_pair(0, 1, 60.0, 0.0)
    eng.step(5, 1)
    orc.step(5, 1)
    assert rel_err(eng.download()["f"], orc.state()["f"]) < 1e-10
    eng.set_thermostat(True)
    eng.step(6, 1)
    assert eng.status() == 0


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_conservative_toggle_follows_the_reference(engine_mod, oracle_mod, precision):
    """ToggleDPDBeadConservativeForces (CNTCell.cpp:235-310): off zeroes every
    a_ij, on restores the tables it saved."""
    s = W.binary_mixture(cells=(6, 7, 8))
    eng, orc = _both(engine_mod, oracle_mod, s, precision)
    tol = 1e-4 if precision == 0 else 1e-10
    eng.step(1, 2)
    orc.step(1, 2)
    eng.set_conservative(False)
    for i in range(2):
        for j in range(i, 2):
            orc.set_pair(i, j, 0.0, s.gamma[i, j])
    eng.step(3, 2)
    orc.step(3, 2)
    assert rel_err(eng.download()["f"], orc.state()["f"]) < tol
    eng.set_conservative(True)
    for i in range(2):
        for j in range(i, 2):
            orc.set_pair(i, j, s.a[i, j], s.gamma[i, j])
    eng.step(5, 2)
    orc.step(5, 2)
    g, o = eng.download(), orc.state()
    assert rel_err(g["f"], o["f"]) < tol
    assert np.array_equal(eng.cells(), orc.cells())
    assert eng.status() == 0


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_renormalised_momenta_follow_the_reference(engine_mod, oracle_mod, precision):
    """CSimBox::UpdateRenormalisedMom (SimBox.cpp:3177-3225) between steps, as
    the reference's Run calls it before Evolve (SimBox.cpp:1314-1317)."""
    s = W.bilayer(cells=(12, 12, 12), nlipids=60)
    s.v *= 1.7          # far from kT = 1, so the rescale is large
    eng, orc = _both(engine_mod, oracle_mod, s, precision)
    eng.step(1, 3)
    orc.step(1, 3)
    eng.renormalise_mom()
    orc.renormalise_mom()
    g, o = eng.download(), orc.state()
    vtol = 1e-5 if precision == 0 else 1e-12
    assert rel_err(g["v"], o["v"], scale=1.0) < vtol
    kT = float((g["v"] ** 2).sum() / (3 * s.n))
    assert abs(kT - s.kT) < 1e-12
    # the renormalised momenta drive the next drift
    eng.step(4, 2)
    orc.step(4, 2)
    g, o = eng.download(), orc.state()
    ftol = 1e-4 if precision == 0 else 1e-10
    assert rel_err(g["f"], o["f"]) < ftol
    assert float(np.max(np.abs(g["unpbc"] - o["unpbc"]))) < (1e-6 if precision == 0 else 1e-12)
    assert eng.status() == 0


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_step_counter_follows_the_calls(engine_mod, oracle_mod, precision):
    """The pair noise is keyed on the step: calls that continue where the
    previous one ended and calls that name another step both draw the noise
    of the steps they name (the device counter is set only on a jump)."""
    s = W.binary_mixture(8)
    eng, orc = _both(engine_mod, oracle_mod, s, precision)
    for t0, k in ((1, 3), (4, 2), (50, 2), (52, 1), (7, 2)):
        eng.step(t0, k)
        orc.step(t0, k)
    ftol = 1e-4 if precision == 0 else 1e-10
    assert rel_err(eng.download()["f"], orc.state()["f"]) < ftol
    assert eng.status() == 0


def test_reuploaded_topology_equals_a_fresh_engine(engine_mod):
    """Re-uploading the same beads and topology (the engine reuses its last
    topology build), a changed topology and changed bead ids (both rebuilt)
    all step exactly as a fresh engine given the same state (full shell:
    bitwise reproducible)."""
    s = W.bilayer(cells=(12, 12, 12), nlipids=60)
    topo = (s.bond_head, s.bond_tail, s.bond_k2, s.bond_l0, s.angle_first, s.angle_second, s.angle_k3,
            s.angle_phi0)

    def run(eng, ids=s.ids, t=topo):
        eng.upload_beads(ids, s.types, s.movable, s.x, s.unpbc, s.v, s.f)
        eng.upload_topology(*t)
        eng.step(1, 4)
        return eng.download()["f"]

    fresh = engine_mod.DpdEngine.from_system(s, precision=1, topology=False)
    want = run(fresh)
    a = engine_mod.DpdEngine.from_system(s, precision=1, topology=False)
    run(a)
    assert np.array_equal(run(a), want)                     # same topology, same ids: reused
    k2 = np.array(s.bond_k2, copy=True)
    k2[::3] *= 1.5
    t2 = (s.bond_head, s.bond_tail, k2) + topo[3:]
    fresh2 = engine_mod.DpdEngine.from_system(s, precision=1, topology=False)
    assert np.array_equal(run(a, t=t2), run(fresh2, t=t2))  # changed spring constants: rebuilt
    assert not np.array_equal(run(a), run(a, t=t2))
    ids = np.asarray(s.ids) + 7                              # other ids, same bonds by id: rebuilt
    t3 = (np.asarray(s.bond_head) + 7, np.asarray(s.bond_tail) + 7) + topo[2:]
    fresh3 = engine_mod.DpdEngine.from_system(s, precision=1, topology=False)
    assert np.array_equal(run(a, ids=ids, t=t3), run(fresh3, ids=ids, t=t3))
    assert a.status() == 0


def test_step_returns_the_fatal_status_without_waiting(engine_mod):
    """A non-finite state raised on the device is returned by a later
    dpd_engine_step (DPD_E_STATUS, no further work queued) without a
    synchronous status call: at most two calls after the step that raised it."""
    s = W.water(6)
    eng = engine_mod.DpdEngine.from_system(s, precision=engine_mod.MIXED)
    f = np.zeros_like(s.x)
    f[10] = [1e308, 0.0, 0.0]
    eng.upload_beads(s.ids, s.types, s.movable, s.x, s.unpbc, s.v, f)
    import torch
    eng.step(1, 1)                       # raises the non-finite bit on the device
    torch.cuda.synchronize()             # the device work has finished; no engine call waited for it
    eng.step(2, 1)                       # its first kernel publishes the status of call 1
    torch.cuda.synchronize()
    with pytest.raises(engine_mod.EngineError, match=r"\(-5\).*non-finite"):
        eng.step(3, 1)
    l0 = eng.launch_count()
    with pytest.raises(engine_mod.EngineError):
        eng.step(3, 1)
    assert eng.launch_count() == l0      # nothing is queued on the invalid state
    # a fresh upload clears the status and the engine steps again
    eng.upload_beads(s.ids, s.types, s.movable, s.x, s.unpbc, s.v)
    eng.step(10, 2)
    eng.step(12, 2)
    assert eng.status() == 0
    eng.close()
