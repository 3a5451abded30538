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


def _snapshot_file(tmp_path):
    from uvlm_b200 import output

    rng = np.random.default_rng(3)
    shapes = [(2, 3, 1.0, 2.0), (2, 3, 1.0, 2.0)]
    n = 12 + 3
    rings = np.round(rng.standard_normal((n, 4, 3)), 3) * [1.0, 1e-7, 1e7]   # exercise %g's exponent form
    g = rng.standard_normal(n)
    path = str(tmp_path / "00000002")
    output.write_legacy_snapshot2(path, 0.5, shapes, rings, rings, g, rng.standard_normal((12, 3)),
                                  rng.standard_normal((12, 4, 3)), np.tile([1.0, 0.0, 0.0], (12, 1)))
    return path, output.read_snapshot2_file(path)


def test_dump_circulation_text(tmp_path):
    """dump_circulation_main.cpp:23-57: 'index i j gamma x y z ...' per ring of every container, a blank line
    per ring row and two more per container; numbers in the C++ stream default (%g)."""
    from uvlm_b200 import tools

    path, snap = _snapshot_file(tmp_path)
    want = []
    for index in range(2):
        for i in range(2):
            for j in range(3):
                k = 6 * index + 3 * i + j
                vals = [snap["gammas"][k], *snap["rings"][k].ravel()]
                want.append("%d\t%d\t%d\t" % (index, i, j) + "\t".join("%g" % v for v in vals) + "\n")
            want.append("\n")
        want.append("\n\n")
    assert tools.dump_circulation(snap) == "".join(want)
    out = str(tmp_path / "circ.dat")
    assert tools.main(["dump_circulation", "--input", path, "--output", out]) == 0
    text = open(out).read()
    assert text == "".join(want) and "e-07" in text and "e+0" in text


def test_dump_centroid_files(tmp_path, capsys):
    """dump_centroid_main.cpp:30-122: <name>_node.dat (closed ring outlines), <name>_cent.dat (centroids) and
    <name>_vel.dat (centroid, morphing-velocity center), and the gnuplot command on stdout."""
    from uvlm_b200 import tools

    path, snap = _snapshot_file(tmp_path)
    d = tmp_path / "dump"
    d.mkdir()
    assert tools.main(["dump_centroid", "--input", path, "--output", str(d)]) == 0
    node = open(d / "00000002_node.dat").read()
    cent = open(d / "00000002_cent.dat").read().splitlines()
    vel = open(d / "00000002_vel.dat").read()
    assert node.count("\n\n\n") == 12 and len(node.split("\n\n\n")[0].splitlines()) == 5
    first = [float(x) for x in node.splitlines()[0].split("\t")]
    np.testing.assert_allclose(first, snap["rings"][0, 0], rtol=1e-5)
    assert len(cent) == 12
    c = snap["rings"][7].sum(0) / 4
    np.testing.assert_allclose([float(x) for x in cent[7].split("\t")], c, rtol=1e-5, atol=1e-12)
    rows = vel.rstrip("\n").splitlines()
    assert vel.endswith("\n\n\n") and len(rows) == 12
    np.testing.assert_allclose([float(x) for x in rows[3].split("\t")][3:], snap["mv_center"][3], rtol=1e-5)
    assert "splot" in capsys.readouterr().out
    # one morphing record short: no velocity rows (DumpVel returns early)
    snap["mv_center"] = snap["mv_center"][:-1]
    assert tools.dump_centroid(snap)[2] == ""


def test_calc_impulse_rejects_incomplete_snapshots(tmp_path):
    """calc_impulse needs a first container whose rings and morphing records are all in the file (the
    reference indexes them unchecked); the checks run before any GPU call."""
    import pytest

    from uvlm_b200 import output, tools

    empty = str(tmp_path / "e")
    output.write_legacy_snapshot2(empty, 0.0, [], np.zeros((0, 4, 3)), None, [], np.zeros((0, 3)),
                                  np.zeros((0, 4, 3)), np.zeros((0, 3)))
    with pytest.raises(ValueError, match="no container"):
        tools.calc_impulse(output.read_snapshot2_file(empty))
    short = str(tmp_path / "s")
    rings = np.random.default_rng(0).standard_normal((6, 4, 3))
    output.write_legacy_snapshot2(short, 0.0, [(2, 3, 1.0, 1.0)], rings, None, np.ones(6), np.zeros((5, 3)),
                                  np.zeros((5, 4, 3)), np.zeros((5, 3)))
    with pytest.raises(ValueError, match="fewer rings or morphing records"):
        tools.calc_impulse(output.read_snapshot2_file(short))
    assert tools.glob_result(str(tmp_path)) == [empty, short]
