"""MainLoop in stages (B200): the six uvlm_stage_* calls reproduce uvlm_step
bit for bit, the state can be read between stages, and calls out of order
are refused without disturbing the context."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(U, precision):
    kw = dict(solver="gmres_stale", warm_start="extrapolate") if precision == "mixed" else {}
    sim = U.SimpleSimulator(precision=precision, **kw)
    m = U.Morphing().set_plug(0.1, 1.0).set_twist(math.radians(8), 1.0, math.pi / 2)
    sim.AddWing(U.RectGenerator(), m, 1.0, 4.0, 6, 16)
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("RK2")
    return sim


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stages_reproduce_step(precision):
    import uvlm_b200 as U

    dt = 2 * math.pi / 40
    a, b = _sim(U, precision), _sim(U, precision)
    a.begin()
    b.begin()
    for s in range(9):
        ra = a.step(s, dt)
        b.stage_kinematics(s, dt)
        b.stage_assemble()
        b.stage_rhs()
        b.stage_solve()
        mid = b.state()                       # readable between stages: the circulations of this step
        b.stage_loads()
        rb = b.stage_advect()
        np.testing.assert_array_equal(ra, rb)
        sa, sb = a.state(), b.state()
        for k in ("wing_pos", "wing_gamma", "wake_pos", "wake_gamma"):
            np.testing.assert_array_equal(sa[k], sb[k])
        np.testing.assert_array_equal(mid["wing_gamma"], sa["wing_gamma"])
    a.close()
    b.close()


def test_stage_order_is_enforced():
    import uvlm_b200 as U

    dt = 0.1
    sim = _sim(U, "fp64")
    ref = _sim(U, "fp64")
    sim.begin()
    ref.begin()
    with pytest.raises(U.UVLMError, match="expected uvlm_stage_kinematics"):
        sim.stage_assemble()
    sim.stage_kinematics(0, dt)
    with pytest.raises(U.UVLMError, match="expected uvlm_stage_assemble"):
        sim.stage_solve()
    with pytest.raises(U.UVLMError, match="in progress"):
        sim.step(0, dt)
    with pytest.raises(U.UVLMError, match="in progress"):
        sim.erase_oldest_wake()
    # the refused calls left the staged step intact: finish it and compare with a plain step
    sim.stage_assemble()
    sim.stage_rhs()
    sim.stage_solve()
    sim.stage_loads()
    np.testing.assert_array_equal(sim.stage_advect(), ref.step(0, dt))
    np.testing.assert_array_equal(sim.step(1, dt), ref.step(1, dt))
    with pytest.raises(U.UVLMError):
        sim.stage_kinematics(2, -1.0)   # dt must be positive; no stage starts
    np.testing.assert_array_equal(sim.step(2, dt), ref.step(2, dt))
    sim.close()
    ref.close()
