"""The oracle reproduces its committed golden fixtures (regression guard).

The fixtures in tests/golden/ were written by tests/golden/make_golden.py;
re-running the oracle must give the same loads and final state to within
the rounding of OpenMP reduction order.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import CASES, run_oracle  # noqa: E402

SMALL = [n for n in CASES if n != "plunge_euler_8x16_200"]


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_fixture(name):
    fx = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    loads, st = run_oracle(CASES[name])
    np.testing.assert_allclose(loads, fx["loads"], rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(st["wing_gamma"], fx["wing_gamma"], rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(st["wake_pos"], fx["wake_pos"], rtol=1e-11, atol=1e-13)


def test_plunge_8x16_fixture_shape_and_physics():
    fx = np.load(os.path.join(HERE, "golden", "plunge_euler_8x16_200.npz"))
    loads = fx["loads"]
    assert loads.shape == (201, 3)
    np.testing.assert_allclose(loads[:, 0], np.arange(201) * 0.125)
    assert fx["wake_gamma"].shape == (1, 200, 16)
    assert fx["wake_pos"].shape == (1, 201, 17, 3)
    # plunge at 5 degrees: mean lift positive, CL oscillates with the heave period (4 s = 32 steps)
    assert loads[40:, 2].mean() > 0.2
    # span mirror symmetry holds up to the rounding that wake roll-up amplifies
    g = fx["wing_gamma"][0]
    np.testing.assert_allclose(g, g[:, ::-1], rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("name", ["plunge_euler_8x16_200", "rk2_heave_pitch_4x8", "rk4_flap_4x8", "ab2_plunge_4x8",
                                  "two_wings_euler_3x6", "erase_euler_4x8"])
def test_sliced_mainloop_and_threaded_lu_are_bit_identical(name):
    """The reference arm's MainLoop cut into slices, with a multithreaded
    FullPivLU, performs exactly MainLoop(step, dt) of the single-threaded
    oracle: the same load rows and the same state, bit for bit."""
    import pyoracle as o

    case = CASES[name]

    def make():
        sim = o.Simulator()
        for w in case["wings"]:
            sim.add_wing(w["chord"], w["span"], w["rows"], w["cols"], origin=w["origin"],
                         kin=o.kinematics(**w["kin"]))
        sim.set_forward_flight(case["ff"])
        sim.set_advection(case["advection"])
        if case.get("erase_wake_after"):
            sim.set_erase_wake_after(case["erase_wake_after"])
        sim.begin()
        return sim

    a, b = make(), make()
    b.set_lu_threads(4)
    for s in range(min(case["steps"], 25) + 1):
        ra = a.step(s, case["dt"])
        k = 1 + s % 7
        b.sliced_begin(s, case["dt"], k, 8)
        rb = np.zeros_like(ra)
        for q in range(k):
            b.sliced_run(q, rb)
        np.testing.assert_array_equal(ra, rb)
    sa, sb = a.state(), b.state()
    for key in sa:
        np.testing.assert_array_equal(sa[key], sb[key])
