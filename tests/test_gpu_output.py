"""Per-step state output of the time-stepper (B200): the records hold the
state after each step's solve (simple_simulator.cpp:270-277): the wing and
its circulations as the step leaves them, the wake after that step's shed
(its newest node row is the trailing edge, the rest is the previous step's
advected wake) and before its advection."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sheet_and_snapshot_records_follow_the_run(tmp_path, precision):
    import uvlm_b200 as U
    from uvlm_b200 import output

    sheets, result = str(tmp_path / "sheets.rec"), str(tmp_path / "result.rec")
    sim = U.SimpleSimulator(precision=precision)
    sim.AddWing(U.RectGenerator(), U.Morphing().set_plug(0.1, 1.0).set_alpha(0.05), 1.0, 4.0, 4, 8)
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("RK2")
    sim.set_sheet_path(sheets)
    sim.set_result_path(result)
    dt = 2 * math.pi / 40
    sim.begin()
    states = []
    for s in range(7):
        sim.step(s, dt)
        states.append(sim.state())
    sim.flush_output()
    recs = output.read_sheets(sheets)
    snaps = output.read_snapshots(result)
    sim.close()
    assert len(recs) == len(snaps) == 7
    for s, rec in enumerate(recs):
        st = states[s]
        assert rec["t"] == s * dt
        pos, g = output.sheet_to_grid(rec["wing"])
        np.testing.assert_array_equal(pos, st["wing_pos"])
        np.testing.assert_array_equal(g, st["wing_gamma"])
        wk = rec["wake"]
        assert wk["num"] == 1 and wk["rows"] == s and wk["cols"] == 8
        wpos, wg = output.sheet_to_grid(wk)
        np.testing.assert_array_equal(wg, st["wake_gamma"])
        if s > 0:
            np.testing.assert_array_equal(wpos[:, 0], st["wing_pos"][:, -1])         # shed trailing edge
            np.testing.assert_array_equal(wpos[:, 1:], states[s - 1]["wake_pos"])   # advected last step
        snap = snaps[s]
        np.testing.assert_array_equal(snap["gammas"], np.concatenate([g.ravel(), wg.ravel()]))
        np.testing.assert_array_equal(snap["rings"][0], [pos[0, 1, 0], pos[0, 1, 1], pos[0, 0, 1], pos[0, 0, 0]])


def test_output_error_paths_and_reopen(tmp_path):
    import uvlm_b200 as U
    from uvlm_b200 import output

    sim = U.SimpleSimulator(precision="fp64")
    sim.AddWing(U.RectGenerator(), U.Morphing().set_plug(0.1, 1.0), 1.0, 4.0, 2, 4)
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    with pytest.raises(U.UVLMError):
        sim.set_sheet_path(str(tmp_path / "no_such_dir" / "x.rec"))   # cannot open: an error, no writer
    sim._sheet_path = None
    sim.flush_output()                                                  # nothing to flush
    first, second = str(tmp_path / "a.rec"), str(tmp_path / "b.rec")
    sim.set_sheet_path(first)
    sim.begin()
    for s in range(3):
        sim.step(s, 0.1)
    sim.set_sheet_path(second)                                          # closes a.rec after its 3 records
    for s in range(3, 5):
        sim.step(s, 0.1)
    sim.close()                                                         # flushes b.rec
    assert [r["t"] for r in output.read_sheets(first)] == [0.0, 0.1, 0.2]
    assert [round(r["t"], 12) for r in output.read_sheets(second)] == [0.3, 0.4]
