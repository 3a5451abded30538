"""Velocity-field tools without a GPU: grid orders of the reference tools and
the wake-front tracker on records written by the library's encoder."""
import ctypes as C

import numpy as np


def test_plane_and_volume_point_orders():
    from uvlm_b200 import tools

    p = tools.plane_points("xz", (-1, 1, 0, 2), 0.5, 3)   # 2d_velocity_main.cpp:58-89: x outer, then y, then z
    assert p.shape == (9, 3)
    np.testing.assert_array_equal(p[:3], [[-1, 0.5, 0], [-1, 0.5, 1], [-1, 0.5, 2]])
    np.testing.assert_array_equal(p[3], [0, 0.5, 0])
    q = tools.volume_points(0, 1, 0, 1, 0, 1, 2)          # 3d_velocity_main.cpp:35-51: z outer, x inner
    np.testing.assert_array_equal(q[:3], [[0, 0, 0], [1, 0, 0], [0, 1, 0]])


def test_wakefront(tmp_path):
    from uvlm_b200 import tools
    from uvlm_b200._capi import check, lib

    P = C.POINTER(C.c_double)
    path = str(tmp_path / "sheets.rec")
    num, rows, cols = 2, 2, 3
    for k, wr in enumerate([0, 1, 2, 3]):
        pos = np.zeros((num, rows + 1, cols + 1, 3))
        g = np.zeros((num, rows, cols))
        wpos = np.zeros((num, wr + 1, cols + 1, 3))
        wpos[..., 0] = 10 * np.arange(num)[:, None, None] + np.arange(wr + 1)[None, :, None] + 0.01 * np.arange(
            cols + 1)[None, None, :]
        wg = np.ones((num, wr, cols))
        check(lib().uvlm_write_state_record(path.encode(), int(k > 0), 0, num, rows, cols, wr, pos.ctypes.data_as(P),
                                            g.ctypes.data_as(P), wpos.ctypes.data_as(P),
                                            wg.ctypes.data_as(P) if wg.size else None, 0.1 * k))
    out = tools.wakefront(path, start=1, wing_id=1)
    # rows - start - 1 >= 0 from the record with 2 wake rows on; row 0 of wing 1: node 0 x of each ring, then node 1
    assert len(out) == 2
    t, *xs = out[0]
    assert t == 0.2
    np.testing.assert_allclose(xs, [10.0, 10.01, 10.02, 10.03])  # node 1 of ring (i, j) is p(i, j+1)
