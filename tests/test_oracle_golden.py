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
