"""Impulse post-processing on the GPU (src/calc_impulse.h, src/calc_impulse_main.cpp) against the oracle.

The reference's own known answers (test/vortex_test.cpp:194-199,
test/calc_impulse_test.cpp:6-52) through the C-ABI, then seeded random wings
with a wake: the vortex impulse of the bound and wake rings and the
Lamb-vector term with every ring inducing velocity at the segment midpoints,
FP64 within 1e-11 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SQUARE2 = np.array([[0, 0, 0], [2, 0, 0], [2, 2, 0], [0, 2, 0]], dtype=float)  # GetSquareRing(2), testutil.h:23-30


def test_kat_ring_impulse():  # test/vortex_test.cpp:194-199
    from uvlm_b200 import rings

    np.testing.assert_allclose(rings.CalcVortexImpulse(SQUARE2[None], [10.0]), [0, 0, -40], atol=1e-12)


@pytest.mark.parametrize("gamma, v_nodes, expect", [
    (1.0, [[1, 0, 0], [2, 0, 0], [3, 0, 0], [4, 0, 0]], [0, 0, 4]),     # test/calc_impulse_test.cpp:6-20
    (2.0, [[1, 0, 0], [2, 0, 0], [3, 0, 0], [4, 0, 0]], [0, 0, 8]),     # :22-36
    (1.0, [[0, 1, 0], [0, 2, 0], [0, 3, 0], [0, 4, 0]], [0, 0, -4]),    # :38-52
])
def test_kat_lamb_vector_no_other_vortex(gamma, v_nodes, expect):
    from uvlm_b200 import rings

    got = rings.CalcLambVector(SQUARE2[None], [gamma], np.array(v_nodes, float)[None], [0, 0, 0],
                               np.zeros((0, 4, 3)), np.zeros(0))
    np.testing.assert_allclose(got, expect, atol=1e-12)


def _rings_of(pos):
    """(rows+1, cols+1, 3) nodes -> (rows*cols, 4, 3) rings in VortexRing node order."""
    a, b = pos[:-1, :-1], pos[1:, :-1]
    c, d = pos[1:, 1:], pos[:-1, 1:]
    return np.stack([a, b, c, d], axis=2).reshape(-1, 4, 3)


def _wing_and_wake(rng, rows, cols, wake_rows):
    i = np.arange(rows + 1)[:, None]
    j = np.arange(cols + 1)[None, :]
    wing = np.zeros((rows + 1, cols + 1, 3))
    wing[..., 0] = 0.25 * i + 0.01 * rng.standard_normal((rows + 1, cols + 1))
    wing[..., 1] = 0.125 * j
    wing[..., 2] = 0.05 * np.sin(0.7 * i + 0.3 * j)
    k = np.arange(wake_rows + 1)[:, None]
    wake = np.zeros((wake_rows + 1, cols + 1, 3))
    wake[..., 0] = 0.25 * rows + 0.2 * k + 0.02 * rng.standard_normal((wake_rows + 1, cols + 1))
    wake[..., 1] = 0.125 * j
    wake[..., 2] = 0.1 * np.sin(0.5 * k) + 0.01 * rng.standard_normal((wake_rows + 1, cols + 1))
    return _rings_of(wing), _rings_of(wake)


@pytest.mark.parametrize("rows, cols, wake_rows", [(1, 2, 0), (4, 8, 6), (7, 33, 21)])
def test_impulse_terms_match_oracle(rows, cols, wake_rows):
    import oracle.pyoracle as o
    from uvlm_b200 import rings

    rng = np.random.default_rng(rows * 100 + cols)
    bound, wake = _wing_and_wake(rng, rows, cols, wake_rows)
    gb = rng.standard_normal(len(bound))
    gw = rng.standard_normal(len(wake))
    allr = np.concatenate([bound, wake]) if len(wake) else bound
    allg = np.concatenate([gb, gw])
    v_nodes = 0.3 * rng.standard_normal((len(bound), 4, 3))
    fs = np.array([-1.0, 0.0, 0.05])

    for r, g in ((bound, gb), (wake, gw)):
        want = o.vortex_impulse(r, g)
        got = rings.CalcVortexImpulse(r, g)
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-12 * max(1.0, np.abs(want).max()))

    # one freestream for all panels, then one per panel (calc_impulse_main.cpp:79-82)
    for f in (fs, fs + 0.01 * rng.standard_normal((len(bound), 3))):
        want = o.lamb_vector(bound, gb, v_nodes, f, allr, allg)
        got = rings.CalcLambVector(bound, gb, v_nodes, f, allr, allg)
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-11 * max(1.0, np.abs(want).max()))


def test_empty_inputs():
    from uvlm_b200 import rings

    assert np.all(rings.CalcVortexImpulse(np.zeros((0, 4, 3)), np.zeros(0)) == 0)
    assert np.all(rings.CalcLambVector(np.zeros((0, 4, 3)), np.zeros(0), np.zeros((0, 4, 3)), [1, 0, 0],
                                       SQUARE2[None], [1.0]) == 0)
