"""dpd_engine_write_restart against the reference's own restart files
(tests/golden/restart_*.npz): an FP64 engine holding the reference's state
writes the bead section of CRestartState::Serialize byte for byte; after
steps, the file parses back to the engine's downloaded state at the format's
6 significant digits."""
import numpy as np
import pytest

from golden_restart import CASES, load_case
from test_restart_format import bead_section

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(CASES))
def test_restart_bead_section_equals_reference(engine_mod, name, tmp_path):
    s, g = load_case(name)
    eng = engine_mod.DpdEngine.from_system(s, precision=1)
    eng.set_restart_layout_for(s)
    path = tmp_path / "dmpcrs.con.dat"
    eng.write_restart(str(path))
    assert path.read_bytes() == bead_section(g["restart"])


@pytest.mark.parametrize("precision", [0, 1], ids=["mixed", "fp64"])
def test_restart_after_steps_parses_to_the_state(engine_mod, tmp_path, precision):
    s, _ = load_case("restart_bilayer_6")
    eng = engine_mod.DpdEngine.from_system(s, precision=precision)
    eng.set_restart_layout_for(s)
    eng.step(1, 7)
    path = tmp_path / "r.dat"
    eng.write_restart(str(path), wall=False, gravity=False, shear=False)
    lines = path.read_text().splitlines()
    assert lines[0] == "0 0 0" and len(lines) == s.n + 1
    rec = np.array([[float(t) for t in ln.split()] for ln in lines[1:]])
    assert np.array_equal(rec[:, 2].astype(np.int64), s.ids)
    assert np.array_equal(rec[:, 3].astype(np.int32), s.types)
    gs = eng.download()
    x = gs["x"].copy()
    x[(x < 0.001)] = 0.001
    for cols, ref in ((slice(5, 8), x), (slice(8, 11), gs["unpbc"]), (slice(11, 14), gs["v"]), (slice(14, 17), gs["f"])):
        assert np.allclose(rec[:, cols], ref, rtol=1e-5, atol=1e-5)


def test_restart_needs_a_layout(engine_mod, tmp_path):
    s, _ = load_case("restart_polymer_6")
    eng = engine_mod.DpdEngine.from_system(s, precision=1)
    with pytest.raises(engine_mod.EngineError):
        eng.write_restart(str(tmp_path / "r.dat"))
    eng.set_restart_layout_for(s)
    eng.upload_beads(s.ids, s.types, s.movable, s.x, s.unpbc, s.v, s.f)
    with pytest.raises(engine_mod.EngineError):
        eng.write_restart(str(tmp_path / "r.dat"))   # cleared by the upload
