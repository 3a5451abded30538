"""Host-side wing lattice generators (uvlm_b200.wing) against the oracle's
restatement of src/wing/*: the same points bit for bit, for every generator
and spacing, and the whole-wing mirror order of src/wing/wing.cpp:12-52.
Also checks that the benchmark workloads and the full-size fixture cases
describe the same set-ups."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import pyoracle as o  # noqa: E402

from uvlm_b200 import wing as W  # noqa: E402


@pytest.mark.parametrize("gen,digit", [("rect", 0), ("naca4digit", 83), ("naca4digit", 2412), ("naca00xx", 12)])
@pytest.mark.parametrize("cheb", [(False, False), (True, False), (False, True), (True, True)])
def test_generators_match_oracle(gen, digit, cheb):
    chord, span, rows, cols = 1.3, 2.5, 7, 9
    g = {"rect": lambda: W.RectGenerator(*cheb), "naca4digit": lambda: W.NACA4digitGenerator(digit, *cheb),
         "naca00xx": lambda: W.NACA00XXGenerator(digit, *cheb)}[gen]()
    got = g.Generate(chord, span, rows, cols)
    ref = o.generate_wing(gen, digit, chord, span, rows, cols, *cheb)
    np.testing.assert_array_equal(got, ref)


def test_whole_wing_matches_oracle():
    half = W.NACA4digitGenerator(83).Generate(1.0, 3.0, 4, 5)
    origin = (0.5, -1.0, 0.25)
    ref = o.whole_wing(half, 4, 5, origin)
    got = W.WholeWing(half, origin)
    assert got.shape == (5, 11, 3)
    np.testing.assert_array_equal(got.reshape(-1, 3), np.asarray(ref).reshape(-1, 3))
    # mirror order: row i is the reversed mirror image, then the half without its first node
    np.testing.assert_array_equal(got[:, 5, 1], np.full(5, origin[1]))
    np.testing.assert_array_equal(got[:, 0, 1], -half[:, -1, 1] + origin[1])


def test_naca_functions_match_oracle():
    for x in np.linspace(0, 1, 37):
        assert W.NACA4digit(x, 1.0, 83) == o.naca4digit(x, 1.0, 83)
        assert W.NACA00XX(x, 1.0, 12) == o.naca00xx(x, 1.0, 12)


def test_bench_workloads_match_fullsize_cases():
    sys.path.insert(0, ROOT)
    import bench
    from cases import FULLSIZE

    for name, wl_name in [("heave_pitch_32x128", "heave_pitch"), ("tandem4_16x64", "tandem4"),
                          ("morphing_24x96", "morphing")]:
        wl, case = bench.WORKLOADS[wl_name](), FULLSIZE[name]
        assert wl.dt == case["dt"] and wl.advection == case["advection"]
        assert len(wl.wings) == len(case["wings"])
        for a, b in zip(wl.wings, case["wings"]):
            for k in ("chord", "span", "rows", "cols"):
                assert a[k] == b[k]
            assert tuple(a["origin"]) == tuple(b["origin"])
            for k in set(a["kin"]) | set(b["kin"]):
                assert a["kin"].get(k, 0.0) == b["kin"].get(k, 0.0), (name, k)
