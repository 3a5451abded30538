"""Known-answer tests that pin the CPU oracle to the reference's own gtests.

Each test restates one case of xeno14/UVLM's gtest suite (file:line given),
with the same inputs, expected values and tolerances.  The oracle
(oracle/uvlm_oracle.cpp) is what every CUDA parity test compares against, so these
are the pins that make it trustworthy.
"""
import math
import os

import numpy as np
import pytest

import pyoracle as o

EPS = 1e-10
SQ2 = math.sqrt(2.0)


def square_ring(l, x0=None, y0=None):
    """test/testutil.h:23-46 (GetSquareRing)."""
    if x0 is None:
        return np.array([[0, 0, 0], [l, 0, 0], [l, l, 0], [0, l, 0]], float)
    x0 -= l / 2
    y0 -= l / 2
    return np.array([[x0, y0, 0], [x0 + l, y0, 0], [x0 + l, y0 + l, 0], [x0, y0 + l, 0]], float)


def assert_double_eq(expected, actual):
    """gtest EXPECT_DOUBLE_EQ: equal within 4 ULPs."""
    expected = np.asarray(expected, float)
    actual = np.asarray(actual, float)
    tol = 4 * np.spacing(np.maximum(np.abs(expected), np.abs(actual)))
    assert np.all(np.abs(expected - actual) <= tol), (expected, actual)


# ---------------------------------------------------------- test/vortex_test.cpp
def test_distance_line_and_point():  # vortex_test.cpp:16-28
    assert abs(o.distance_line_and_point([0, 0, -1], [0, 0, 1], [1, 0, 0]) - 1) < EPS
    assert abs(o.distance_line_and_point([0, 0, 0], [1, 1, 0], [1, 0, 0]) - SQ2 / 2) < EPS


@pytest.mark.parametrize("x,expected", [(1, 1 / 2 / math.pi), (2, 1 / 4 / math.pi), (8, 1 / 16 / math.pi)])
def test_biot_savart_infinite_length(x, expected):  # vortex_test.cpp:34-49
    r = o.biot_savart([0, 0, -1e10], [0, 0, 1e10], [x, 0, 0])
    np.testing.assert_allclose(r, [0, expected, 0], atol=EPS, rtol=0)


def test_biot_savart_finite_length():  # vortex_test.cpp:51-59
    r = o.biot_savart([0, 0, -1], [0, 0, 1], [1, 0, 0])
    np.testing.assert_allclose(r, [0, SQ2 / 4 / math.pi, 0], atol=EPS, rtol=0)


def test_biot_savart_midpoint_cutoff():  # vortex_test.cpp:61-67
    a = np.array([SQ2, 2, math.pi])
    b = np.array([100, 2121, 12434.0])
    assert np.linalg.norm(o.biot_savart(a, b, (a + b) / 2)) < EPS


def test_biot_savart_endpoint_cutoff():  # vortex_test.cpp:69-79
    a = np.array([math.pi, SQ2, -1])
    b = np.array([0, 0, 1.0])
    assert np.linalg.norm(o.biot_savart(a, b, a)) < EPS
    assert np.linalg.norm(o.biot_savart(a, b, b)) < EPS


RING_2 = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], float)


def test_ring_biot_savart():  # vortex_test.cpp:104-116
    assert_double_eq([0, 0, -4 * SQ2], o.ring_biot_savart(RING_2, 4 * math.pi, [0, 0, 0]))


def test_ring_chordwise_biot_savart():  # vortex_test.cpp:118-130
    assert_double_eq([0, 0, -2 * SQ2], o.ring_biot_savart(RING_2, 4 * math.pi, [0, 0, 0], chordwise=True))


def test_ring_normal_and_tangents():  # vortex_test.cpp:132-167
    sq = square_ring(20000)
    assert_double_eq([0, 0, 1], o.ring_vector(sq, "normal"))
    lean = np.array([[0, 0, 0], [1, 0, 1], [1, 1, 1], [0, 1, 0]], float)
    assert_double_eq([-math.sqrt(0.5), 0, math.sqrt(0.5)], o.ring_vector(lean, "normal"))
    assert_double_eq([1, 0, 0], o.ring_vector(sq, "tangent"))
    lean2 = np.array([[0, 0, 0], [1, 0, 0.5], [1, 1, 0.5], [0, 1, 0]], float)
    assert_double_eq([2 / math.sqrt(5), 0, 1 / math.sqrt(5)], o.ring_vector(lean2, "tangent"))
    assert_double_eq([0, 1, 0], o.ring_vector(sq, "tangent2"))


def test_ring_angle_of_attack():  # vortex_test.cpp:169-174
    alpha = 0.1
    assert_double_eq(alpha, o.ring_angle_of_attack(square_ring(1), [math.cos(alpha), 0, math.sin(alpha)]))


def test_ring_impulse():  # vortex_test.cpp:194-199
    assert_double_eq([0, 0, -40], o.ring_vector(square_ring(2), "impulse", gamma=10))


def test_ring_chord_span_area():  # vortex_test.cpp:201-232
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 2.1, 0], [0, 2, 0]], float)
    assert_double_eq([1, 0, 0], o.ring_vector(v, "tanvec_chord"))
    assert_double_eq([0, 1, 0], o.ring_vector(v, "tanvec_span"))
    assert_double_eq(1, o.ring_scalar(v, "c"))
    assert_double_eq(2, o.ring_scalar(v, "b"))
    assert abs(o.ring_scalar(v, "area") - 2.05) < EPS


def test_ring_segment_orientation():  # vortex_test.cpp:176-192 (ForEachSegment)
    # ForEachSegment walks start=nodes[k+1] -> end=nodes[k]; with unit Gamma the
    # ring velocity equals the sum of those four Biot-Savart segments.
    sq = square_ring(1)
    x = np.array([0.3, 0.2, 0.7])
    expected = sum(o.biot_savart(sq[(k + 1) % 4], sq[k], x) for k in range(4))
    np.testing.assert_allclose(o.ring_biot_savart(sq, 1.0, x), expected, rtol=0, atol=1e-15)


# ------------------------------------------------------------ test/shed_test.cpp
SHED_RING = np.array([[1, 1, 0], [-1, 1, 0], [-1, -1, 0], [1, -1, 0]], float)


def test_induced_velocity_many_rings():  # shed_test.cpp:21-35
    n = 20
    rings = np.stack([SHED_RING] * n)
    res = o.rings_induced_velocity(rings, np.full(n, 4 * math.pi), [0, 0, 0])
    assert_double_eq([0, 0, -4 * SQ2 * n], res)


def test_chordwise_induced_velocity_many_rings():  # shed_test.cpp:37-50
    n = 20
    rings = np.stack([SHED_RING] * n)
    res = o.rings_induced_velocity(rings, np.full(n, 4 * math.pi), [0, 0, 0], chordwise=True)
    assert_double_eq([0, 0, -4 * SQ2 / 2 * n], res)


def test_connect_trailing_edge():  # shed_test.cpp:52-65
    edge = np.stack([square_ring(2, 1, 1), square_ring(2, 1, 3)])
    wake = np.stack([square_ring(2, 99, 1), square_ring(2, 99, 3)])
    w = o.connect_trailing_edge(edge, wake)
    assert_double_eq([[2, 0, 0], [100, 0, 0], [100, 2, 0], [2, 2, 0]], w[0])
    assert_double_eq([[2, 2, 0], [100, 2, 0], [100, 4, 0], [2, 4, 0]], w[1])


@pytest.mark.parametrize("parallel", [False, True])
def test_advect_no_vortex(parallel):  # shed_test.cpp:67-91
    wake = square_ring(2, 0, 0)[None]
    w = o.rings_advect(np.zeros((0, 4, 3)), np.zeros(0), wake, [1, 0, 0], 0.1, parallel=parallel)
    assert_double_eq([[-1 + 0.1, -1, 0], [1 + 0.1, -1, 0], [1 + 0.1, 1, 0], [-1 + 0.1, 1, 0]], w[0])


# ----------------------------------------------------------- test/linear_test.cpp
def test_calc_morphing_velocity_flap():  # linear_test.cpp:27-49
    kin = o.kinematics(flap_amp=1.0, flap_omega=1.0)  # flap(t) = sin(t)
    panels = np.stack([square_ring(1, 0, 1), square_ring(1, 0, -2)])
    assert_double_eq([0, 0, 1], o.ring_vector(panels[0], "normal"))
    assert_double_eq([0, 1, 0], o.ring_vector(panels[0], "centroid"))
    assert_double_eq([0, -2, 0], o.ring_vector(panels[1], "centroid"))
    res = o.calc_morphing_velocity_on_wing(panels, kin, 0.0)
    assert abs(res[0] - 1) < EPS
    assert abs(res[1] - 2) < EPS


def test_solve_linear_no_wake():  # linear_test.cpp:61-81
    alpha, U, a = math.pi / 6, 2.0, 0.1
    v = np.array([[0, 0, 0], [a * math.cos(alpha), 0, -a * math.sin(alpha)],
                  [a * math.cos(alpha), a, -a * math.sin(alpha)], [0, a, 0]])
    g = o.solve_linear_problem(v[None], np.zeros((0, 4, 3)), np.zeros(0), [U, 0, 0], o.Kinematics(), 0.0)
    assert abs(g[0] - SQ2 * math.pi * a * U * math.sin(alpha) / 4) < EPS


def _two_rings():
    return np.stack([square_ring(2, -1, 0), square_ring(2, 1, 0)])


def test_solve_linear_no_wake_no_morphing():  # linear_test.cpp:83-98
    vs = _two_rings()
    g = o.solve_linear_problem(vs, np.zeros((0, 4, 3)), np.zeros(0), [0, 0, 1], o.Kinematics(), 0.0)
    for x in ([-1, 0, 0], [1, 0, 0]):
        assert_double_eq([0, 0, -1], o.rings_induced_velocity(vs, g, x))


def test_solve_linear_no_wake_morphing():  # linear_test.cpp:100-116
    vs = _two_rings()
    kin = o.kinematics(plug_amp=0.1, plug_omega=1.0)  # plug(t) = 0.1 sin(t)
    g = o.solve_linear_problem(vs, np.zeros((0, 4, 3)), np.zeros(0), [0, 0, 1], kin, 0.0)
    for x in ([-1, 0, 0], [1, 0, 0]):
        np.testing.assert_allclose(o.rings_induced_velocity(vs, g, x), [0, 0, -1 + 0.1], atol=EPS, rtol=0)


def test_solve_linear_wake_term_is_dropped_like_reference():
    # linear_test.cpp:118-139 exercises src/linear.inl:113-130, whose wake RHS
    # term is a discarded statement (:123-124), so the wake has no effect on
    # the solution.  The oracle reproduces that; with the term enabled the
    # wake-induced normal wash is subtracted instead.
    vs = _two_rings()
    wake = square_ring(2, 2, 0)[None]
    kin = o.kinematics(plug_amp=0.1, plug_omega=1.0)
    g_ref = o.solve_linear_problem(vs, wake, [1.0], [0, 0, 1], kin, 0.0, drop_wake_term=True)
    g_none = o.solve_linear_problem(vs, np.zeros((0, 4, 3)), np.zeros(0), [0, 0, 1], kin, 0.0)
    np.testing.assert_array_equal(g_ref, g_none)
    g_fix = o.solve_linear_problem(vs, wake, [1.0], [0, 0, 1], kin, 0.0, drop_wake_term=False)
    for x in ([-1, 0, 0], [1, 0, 0]):
        w = o.rings_induced_velocity(wake, [1.0], x)
        np.testing.assert_allclose(o.rings_induced_velocity(vs, g_fix, x), [0, 0, -1 + 0.1 - w[2]],
                                   atol=EPS, rtol=0)


# --------------------------------------------------------- test/morphing_test.cpp
MEPS = 1e-6


def _near(x, y, eps=MEPS):
    np.testing.assert_allclose(x, y, atol=eps, rtol=0)


def test_perfome_plug():  # morphing_test.cpp:24-43
    k = o.kinematics(plug_amp=1, plug_omega=1)
    _near(o.perfome(k, [1, 0, 0], 0), [1, 0, 0])
    _near(o.perfome(k, [2, 0, 0], 0), [2, 0, 0])
    _near(o.perfome(k, [1, 0, 0], math.pi / 2), [1, 0, 1])


def test_perfome_plug_origin():  # morphing_test.cpp:45-66
    k = o.kinematics(plug_amp=1, plug_omega=1, origin=(1, 2, 3))
    _near(o.perfome(k, [2, 2, 3], 0), [2, 2, 3])
    _near(o.perfome(k, [3, 2, 3], 0), [3, 2, 3])
    _near(o.perfome(k, [2, 2, 3], math.pi / 2), [2, 2, 4])


def test_perfome_flap():  # morphing_test.cpp:68-82 (flap = pi/4 cos t)
    k = o.kinematics(flap_amp=math.pi / 4, flap_omega=1, flap_phase=math.pi / 2)
    _near(o.perfome(k, [0, 1, 0], 0), [0, math.sqrt(0.5), math.sqrt(0.5)])
    _near(o.perfome(k, [0, 1, 0], math.pi / 2), [0, 1, 0])


def test_perfome_flap_origin():  # morphing_test.cpp:84-98
    k = o.kinematics(flap_amp=math.pi / 4, flap_omega=1, flap_phase=math.pi / 2, origin=(0, 1, 0))
    _near(o.perfome(k, [0, 2, 0], 0), [0, 1 + math.sqrt(0.5), math.sqrt(0.5)])
    _near(o.perfome(k, [0, 2, 0], math.pi / 2), [0, 2, 0])


def test_morphing_velocity_plug():  # morphing_test.cpp:118-143
    k = o.kinematics(plug_amp=1, plug_omega=1)
    _near(o.morph_velocity(k, [1, 0, 0], 0), [0, 0, 1])
    _near(o.morph_velocity(k, [2, 0, 0], 0), [0, 0, 1])
    _near(o.morph_velocity(k, [1, 0, 0], math.pi / 2), [0, 0, 0])
    _near(o.morph_velocity(k, [1, 2, 3], math.pi / 4), [0, 0, math.sqrt(0.5)])


def test_morphing_velocity_plug2():  # morphing_test.cpp:145-153
    k = o.kinematics(plug_amp=0.175, plug_omega=1)
    _near(o.morph_velocity(k, [100, 2000, 3333], 0), [0, 0, 0.175])


# -------------------------------------------------------- test/calc_load_test.cpp
def test_calc_um():  # calc_load_test.cpp:37-46
    k = o.kinematics(plug_amp=1, plug_omega=1)
    np.testing.assert_allclose(o.calc_um(k, [0, 0, 0], [1, 0, 0], 0), [1, 0, -1], atol=EPS, rtol=0)
    np.testing.assert_allclose(o.calc_um(k, [0, 0, 0], [1, 0, 0], math.pi / 3), [1, 0, -0.5], atol=EPS,
                               rtol=0)


# ---------------------------------------------------- test/wing_test.cpp, rect_test
def test_whole_wing_mirror():  # wing_test.cpp:30-43
    half = o.rect_generate(1, 2, 2, 2)
    pos = o.whole_wing(half, 2, 2)
    assert pos.shape == (15, 3)
    for k, e in [(0, (0, -2, 0)), (1, (0, -1, 0)), (2, (0, 0, 0)), (3, (0, 1, 0)), (4, (0, 2, 0)),
                 (5, (0.5, -2, 0)), (10, (1, -2, 0)), (14, (1, 2, 0))]:
        np.testing.assert_allclose(pos[k], e, atol=EPS, rtol=0)


def test_whole_wing_origin():  # wing_test.cpp:45-58
    half = o.rect_generate(1, 2, 2, 2)
    pos = o.whole_wing(half, 2, 2, origin=(1, 2, 3))
    for k, e in [(0, (1, 0, 3)), (1, (1, 1, 3)), (2, (1, 2, 3)), (3, (1, 3, 3)), (4, (1, 4, 3)),
                 (5, (1.5, 0, 3)), (10, (2, 0, 3)), (14, (2, 4, 3))]:
        np.testing.assert_allclose(pos[k], e, atol=EPS, rtol=0)


@pytest.mark.parametrize("scale", [1, 2])
def test_transform_chebyshev(scale):  # rect_test.cpp:6-24
    x = o.transform_chebyshev(5, 0, scale)
    assert_double_eq([0, scale * math.cos(-math.pi / 8 * 3), scale * math.cos(-math.pi / 8 * 2),
                      scale * math.cos(-math.pi / 8 * 1), scale], x)


# ------------------------------------------------------- oracle self-consistency
def test_fullpiv_lu_matches_lapack():
    rng = np.random.default_rng(0)
    for n in (1, 5, 37, 120):
        A = rng.standard_normal((n, n)) + n * np.eye(n) * rng.random()
        b = rng.standard_normal(n)
        np.testing.assert_allclose(o.fullpiv_lu_solve(A, b), np.linalg.solve(A, b), rtol=1e-9, atol=1e-11)


def test_fullpiv_lu_needs_full_pivoting():
    # A zero diagonal defeats the unpivoted algorithm; complete pivoting solves it.
    A = np.array([[0.0, 2.0, 1.0], [1.0, 0.0, 3.0], [4.0, 1.0, 0.0]])
    b = np.array([1.0, 2.0, 3.0])
    np.testing.assert_allclose(o.fullpiv_lu_solve(A, b), np.linalg.solve(A, b), rtol=1e-13)


def test_voring_matches_reversed_aos_ring():
    # VORING walks p0->p1->p2->p3 (vortex.cpp:145-160); the AoS ring walks
    # nodes[k+1]->nodes[k] (vortex.h:132-140), so the same node order gives the
    # opposite sign.
    rng = np.random.default_rng(1)
    pos = rng.standard_normal((1, 2, 2, 3))
    gamma = np.array([[[0.7]]])
    x = rng.standard_normal(3)
    v_sheet = o.sheet_induced_velocity(pos, gamma, x[None])[0]
    ring = np.stack([pos[0, 0, 0], pos[0, 0, 1], pos[0, 1, 1], pos[0, 1, 0]])
    np.testing.assert_allclose(v_sheet, -o.ring_biot_savart(ring, 0.7, x), rtol=1e-13, atol=1e-15)


def test_simulator_symmetric_and_finite():
    sim = o.Simulator()
    kin = o.kinematics(alpha=math.radians(5), plug_amp=0.1, plug_omega=math.pi / 2)
    sim.add_wing(1.0, 4.0, 4, 8, kin=kin)
    sim.set_forward_flight([-1, 0, 0])
    loads = sim.run(6, 0.125)
    assert loads.shape == (7, 3)
    assert np.all(np.isfinite(loads))
    s = sim.state()
    g = s["wing_gamma"][0]
    np.testing.assert_allclose(g, g[:, ::-1], rtol=1e-9, atol=1e-12)  # span mirror symmetry
    assert s["wake_gamma"].shape == (1, 6, 8)
    assert s["wake_pos"].shape == (1, 7, 9, 3)
    # steady lift at 5 degrees is positive once the start-up transient decays
    assert loads[-1, 2] > 0


SQUARE2 = np.array([[0, 0, 0], [2, 0, 0], [2, 2, 0], [0, 2, 0]], dtype=float)  # GetSquareRing(2), testutil.h:23-30


def test_kat_ring_impulse():  # test/vortex_test.cpp:194-199
    np.testing.assert_allclose(o.vortex_impulse(SQUARE2[None], [10.0]), [0, 0, -40], atol=1e-12)


@pytest.mark.parametrize("gamma, v_nodes, expect", [
    (1.0, [[1, 0, 0], [2, 0, 0], [3, 0, 0], [4, 0, 0]], [0, 0, 4]),     # test/calc_impulse_test.cpp:6-20
    (2.0, [[1, 0, 0], [2, 0, 0], [3, 0, 0], [4, 0, 0]], [0, 0, 8]),     # :22-36
    (1.0, [[0, 1, 0], [0, 2, 0], [0, 3, 0], [0, 4, 0]], [0, 0, -4]),    # :38-52
])
def test_kat_lamb_vector_no_other_vortex(gamma, v_nodes, expect):
    got = o.lamb_vector(SQUARE2[None], [gamma], np.array(v_nodes, float)[None], [0, 0, 0], np.zeros((0, 12)),
                        np.zeros(0))
    np.testing.assert_allclose(got, expect, atol=1e-12)


def test_katz_plotkin_flat_panel_steady():
    """A steady flat unit panel in U = (1, 0, 0): alpha = 0, L_st = rho U G b, no drag, no Pin
    (CalcLoadKatzPlotkin, src/calc_load/katz_plotkin.cpp:16-68)."""
    k = o.Kinematics()
    out = o.load_katz_plotkin(SQUARE2[None] / 2, [0.7], [0.7], 1, 1, k, [1, 0, 0], 1.0, 0.0, 0.1)
    np.testing.assert_allclose(out, [0, 0, 0.7, 0, 0], atol=1e-14)


def test_wing_builder_mirror_and_build():  # test/wing_builder_test.cpp:31-123
    import legacy_oracle as L

    pts = np.array([[[i, j, 0] for j in range(4)] for i in range(3)], float)  # rows 2, cols 3, p = (i, j, 0)
    r = L.container_rings(pts, 2, 3, (0, 0, 0))
    assert r.shape == (12, 4, 3)                              # 2 x 6 rings
    np.testing.assert_array_equal(r[0, 0], [0, -3, 0])        # container.at(0, 0).nodes()[0]
    np.testing.assert_array_equal(r[0, 1], [1, -3, 0])
    np.testing.assert_array_equal(r[5, 3], [0, 3, 0])         # ring (0, 5): p(0, 6) = (0, 3, 0)
    r2 = L.container_rings(pts, 2, 3, (0, 0, 1))
    assert np.all(r2[..., 2] == 1)                            # add_multiple_wings: origin z = 1


def test_legacy_loop_symmetric_and_finite():
    import legacy_oracle as L

    X, Y = np.meshgrid(np.linspace(0, 1, 3), np.linspace(0, 2, 4), indexing="ij")
    k = o.Kinematics()
    k.alpha, k.plug_amp, k.plug_omega = 0.1, 0.1, 1.0
    w = dict(rows=2, cols=3, points=np.stack([X, Y, 0 * X], -1), origin=(0, 0, 0), chord=1.0, span=2.0)
    for jouk in (False, True):
        rows = L.start([w], [k], [1, 0, 0], 6, 0.1, use_joukowski=jouk)
        assert rows.shape == (7, 6) and np.all(np.isfinite(rows))
        np.testing.assert_allclose(rows[:, 2], 0, atol=1e-12)   # C_y of a symmetric wing
        assert rows[-1, 3] > 0                                  # lift at alpha = 0.1


# ---- wing generators: test/naca4digit_test.cpp, test/naca00XX_test.cpp ----
# The published section tables the reference's tests read (test/wing/data/)
# are kept in tests/golden/naca_tables.npz (tests/golden/make_naca_tables.py).
_NACA = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "naca_tables.npz"))


def test_naca4digit_table():  # naca4digit_test.cpp:31-43 (mean square error below 1e-6)
    d = _NACA["naca62xx"]
    err = np.mean([(y - o.naca4digit(x, 100, 62)) ** 2 for x, y in d])
    assert 1e-6 > err


def test_naca4digit_generator():  # naca4digit_test.cpp:45-55
    pts = o.generate_wing("naca4digit", 83, 3, 2, 10, 10)
    for p in pts.reshape(-1, 3):
        assert p[2] == o.naca4digit(p[0], 3, 83)


def test_naca00xx_table():  # naca00XX_test.cpp:29-38 (sum of squares below 1e-10)
    d = _NACA["naca0012"]
    err = sum((z - o.naca00xx(x, 1.0, 12)) ** 2 for x, z in d)
    assert 1e-10 > err


@pytest.mark.parametrize("digit", [12, 0])
def test_naca00xx_generator(digit):  # naca00XX_test.cpp:40-68 (Generate, GenerateRect)
    pts = o.generate_wing("naca00xx", digit, 2, 2, 2, 2).reshape(-1, 3)
    z1, z2 = (o.naca00xx(1.0, 2.0, 12), o.naca00xx(2.0, 2.0, 12)) if digit else (0.0, 0.0)
    expect = [(0, 0, 0), (0, 1, 0), (0, 2, 0), (1, 0, z1), (1, 1, z1), (1, 2, z1), (2, 0, z2), (2, 1, z2),
              (2, 2, z2)]
    for p, e in zip(pts, expect):
        np.testing.assert_array_equal(p, e)
