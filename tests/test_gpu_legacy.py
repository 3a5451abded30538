"""The legacy AoS path on the GPU against the FP64 oracle (B200).

Morphing::Perfome / Velocity (src/morphing.cpp:23-52), SolveLinearProblem
over containers with per-wing morphings (src/linear.inl:132-157), the two
container load formulations (src/calc_load/katz_plotkin.cpp:16-68,
src/calc_load/joukowski.h:24-104) and the legacy main loop
(src/simulator/simulator.cpp:220-270) restated in oracle/legacy_oracle.py.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _kin(M, seed, origin=(0.0, 0.0, 0.0)):
    rng = np.random.default_rng(seed)
    m = M.Morphing().set_alpha(0.05 + 0.05 * rng.random()).set_plug(0.1, 1.0, rng.random())
    m.set_flap(0.2 * rng.random(), 0.8, rng.random()).set_twist(0.1 * rng.random(), 1.2, 0.3, 0.02)
    m.set_bend(0.05, 0.02, 0.9, 0.1)
    m.set_origin(origin)
    return m


def _okin(o, m):
    k = o.Kinematics()
    for name, _ in type(m.k)._fields_:
        v = getattr(m.k, name)
        if name == "origin":
            for i in range(3):
                k.origin[i] = v[i]
        else:
            setattr(k, name, v)
    return k


def _plate(rows, cols, chord=1.0, span=2.0, seed=0):
    """rows x cols rings of a wavy plate (AoS, ring (i, j) = p(i,j), p(i+1,j), p(i+1,j+1), p(i,j+1))."""
    rng = np.random.default_rng(seed)
    X, Y = np.meshgrid(np.linspace(0, chord, rows + 1), np.linspace(-span / 2, span / 2, cols + 1), indexing="ij")
    P = np.stack([X, Y, 0.03 * np.sin(2 * X + Y)], -1) + 0.002 * rng.standard_normal((rows + 1, cols + 1, 3))
    return np.stack([P[:-1, :-1], P[1:, :-1], P[1:, 1:], P[:-1, 1:]], 2).reshape(-1, 4, 3)


def test_morphing_perfome_and_velocity():
    import pyoracle as o

    import uvlm_b200 as M

    m = _kin(M, 1, origin=(0.3, 0.1, -0.2))
    k = _okin(o, m)
    x0 = np.random.default_rng(2).uniform(-2, 2, (257, 3))
    for t in (0.0, 0.7, 3.1):
        p = m.Perfome(x0, t)
        v = m.Velocity(x0, t)
        pref = np.array([o.perfome(k, x, t) for x in x0])
        vref = np.array([o.morph_velocity(k, x, t) for x in x0])
        np.testing.assert_allclose(p, pref, rtol=0, atol=1e-13)
        np.testing.assert_allclose(v, vref, rtol=0, atol=1e-8)  # central difference, h = 1e-6


@pytest.mark.parametrize("drop", [True, False])
def test_solve_linear_problem_containers(drop):
    import pyoracle as o

    import uvlm_b200 as M
    from uvlm_b200 import rings

    a, b = _plate(3, 6, seed=1), _plate(2, 4, seed=2) + np.array([0.0, 0.0, 0.6])
    bound = np.concatenate([a, b])
    wake = _plate(4, 6, seed=3) + np.array([1.05, 0.0, 0.02])
    wg = np.random.default_rng(4).standard_normal(len(wake)) * 0.1
    ms = [_kin(M, 5), _kin(M, 6)]
    fs = [1.0, 0.0, 0.05]
    got = rings.SolveLinearProblemContainers(bound, [len(a), len(b)], ms, wake, wg, fs, 0.4, drop_wake_term=drop)
    ref = o.solve_linear_problem_containers(bound, [len(a), len(b)], [_okin(o, m) for m in ms], wake, wg, fs, 0.4,
                                            drop)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-9 * np.max(np.abs(ref)))


def test_katz_plotkin_flat_panel_kat():
    import uvlm_b200 as M
    from uvlm_b200 import rings

    sq = np.array([[[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]]], float)
    out = rings.CalcLoadKatzPlotkin(sq, [0.7], [0.7], 1, 1, M.Morphing(), [1, 0, 0], 1.0, 0.0, 0.1)
    np.testing.assert_allclose(out, [0, 0, 0.7, 0, 0], atol=1e-14)


@pytest.mark.parametrize("with_rings", [False, True])
def test_katz_plotkin_matches_oracle(with_rings):
    import pyoracle as o

    import uvlm_b200 as M
    from uvlm_b200 import rings

    rows, cols = 4, 8
    r = _plate(rows, cols, seed=7)
    rng = np.random.default_rng(8)
    g = 0.2 + 0.1 * rng.standard_normal(rows * cols)
    gp = g - 0.01 * rng.standard_normal(rows * cols)
    m = _kin(M, 9)
    kw = {}
    if with_rings:
        wake = _plate(5, cols, seed=10) + np.array([1.05, 0, 0.01])
        kw = dict(bound_rings=r, bound_gammas=g, wake_rings=wake, wake_gammas=0.05 * rng.standard_normal(len(wake)))
    ref = o.load_katz_plotkin(r, g, gp, rows, cols, _okin(o, m), [1.0, 0.0, 0.1], 1.2, 0.5, 0.05,
                              kw.get("bound_rings"), kw.get("bound_gammas"), kw.get("wake_rings"),
                              kw.get("wake_gammas"))
    got = rings.CalcLoadKatzPlotkin(r, g, gp, rows, cols, m, [1.0, 0.0, 0.1], 1.2, 0.5, 0.05, **kw)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * np.max(np.abs(ref)))


def test_container_joukowski_matches_oracle():
    import pyoracle as o

    import uvlm_b200 as M
    from uvlm_b200 import rings

    rows, cols = 4, 8
    r0 = _plate(rows, cols, seed=11)
    m = _kin(M, 12)
    r = m.Perfome(r0.reshape(-1, 3), 0.5).reshape(-1, 4, 3)
    rng = np.random.default_rng(13)
    g = 0.2 + 0.1 * rng.standard_normal(rows * cols)
    gp = g - 0.01 * rng.standard_normal(rows * cols)
    wake = _plate(5, cols, seed=14) + np.array([1.05, 0, 0.01])
    pool = np.concatenate([r, wake])
    pg = np.concatenate([g, 0.05 * rng.standard_normal(len(wake))])
    ref = o.load_joukowski_rings(r, r0, g, gp, rows, cols, _okin(o, m), pool, pg, [1.0, 0.0, 0.1], 1.2, 0.5, 0.05)
    got = rings.CalcLoadJoukowski(r, r0, g, gp, rows, cols, m, pool, pg, [1.0, 0.0, 0.1], 1.2, 0.5, 0.05)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * np.max(np.abs(ref)))


@pytest.mark.parametrize("joukowski", [False, True])
def test_legacy_start_matches_oracle(joukowski):
    """Two wings (the second above the first, its own morphing), 12 steps: the load file rows."""
    import legacy_oracle as L
    import pyoracle as o

    import uvlm_b200 as M
    from uvlm_b200.legacy import LegacySimulator, Wing

    sim = LegacySimulator(use_joukowski=joukowski)
    w1 = Wing.rect(1.0, 2.0, 3, 4)
    w2 = Wing.rect(1.0, 2.0, 3, 4, origin=(0.0, 0.0, 0.8))
    m1, m2 = _kin(M, 21), _kin(M, 22)
    sim.AddWing(w1, m1)
    sim.AddWing(w2, m2)
    sim.SetInlet(1.0, 0.0, 0.0)
    dt = 2 * math.pi / 40
    got = sim.Start(12, dt)
    oks = []
    for w, m in ((w1, m1), (w2, m2)):
        k = _okin(o, m)
        for i in range(3):
            k.origin[i] = w.origin[i]
        oks.append(k)
    wings = [dict(rows=w.rows, cols=w.cols, points=w.points, origin=w.origin, chord=w.chord, span=w.span)
             for w in (w1, w2)]
    ref = L.start(wings, oks, [1.0, 0.0, 0.0], 12, dt, use_joukowski=joukowski)
    assert got.shape == ref.shape == (13, 11)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-8 * np.max(np.abs(ref[:, 1:])))


def test_legacy_snapshot_files_and_calc_impulse(tmp_path):
    """SetOutputPath / SetOutputLoadPath (simulator.cpp:118-200): one Snapshot2 file per step matching the
    oracle's pool, nodes0 and morphing velocities; the load file's rows; then calc_impulse
    (src/calc_impulse_main.cpp) over those files against the oracle's impulse and Lamb-vector sums."""
    import legacy_oracle as L
    import pyoracle as o

    import uvlm_b200 as M
    from uvlm_b200 import output, tools
    from uvlm_b200.legacy import LegacySimulator, Wing

    steps, dt = 6, 2 * math.pi / 40
    sim = LegacySimulator()
    w1 = Wing.rect(1.0, 2.0, 3, 4)
    w2 = Wing.rect(1.0, 2.0, 3, 4, origin=(0.0, 0.0, 0.8))
    m1, m2 = _kin(M, 31), _kin(M, 32)
    sim.AddWing(w1, m1)
    sim.AddWing(w2, m2)
    out_dir = tmp_path / "result"
    out_dir.mkdir()
    load_path = str(tmp_path / "load.tsv")
    sim.SetOutputPath(str(out_dir))
    sim.SetOutputLoadPath(load_path)
    rows = sim.Start(steps, dt)
    oks = []
    for w, m in ((w1, m1), (w2, m2)):
        k = _okin(o, m)
        for i in range(3):
            k.origin[i] = w.origin[i]
        oks.append(k)
    wings = [dict(rows=w.rows, cols=w.cols, points=w.points, origin=w.origin, chord=w.chord, span=w.span)
             for w in (w1, w2)]
    ref = []
    L.start(wings, oks, [1.0, 0.0, 0.0], steps, dt, snapshots=ref)
    files = tools.glob_result(str(out_dir))
    assert [f[-8:] for f in files] == [f"{s:08d}" for s in range(steps + 1)]
    for step, (f, r) in enumerate(zip(files, ref)):
        snap = output.read_snapshot2_file(f)
        assert snap["t"] == dt * step
        assert [(c["rows"], c["cols"], c["id"], c["chord"], c["span"]) for c in snap["container_shapes"]] == [
            (3, 8, 0, 1.0, 2.0), (3, 8, 1, 1.0, 2.0)]
        assert len(snap["rings"]) == 48 + 8 * step
        scale = np.abs(r["rings"]).max()
        np.testing.assert_allclose(snap["rings"], r["rings"], rtol=0, atol=1e-10 * scale)
        np.testing.assert_array_equal(snap["rings0"], r["rings0"])
        np.testing.assert_allclose(snap["gammas"], r["gammas"], rtol=0, atol=1e-8 * np.abs(r["gammas"]).max())
        for k in ("mv_center", "mv_nodes"):
            np.testing.assert_allclose(snap[k], r[k], rtol=0, atol=1e-8)  # central difference, h = 1e-6
        np.testing.assert_array_equal(snap["mv_freestream"], r["mv_freestream"])
        imp = tools.calc_impulse(snap)
        want = L.calc_impulse(snap)
        np.testing.assert_allclose(imp, want, rtol=0, atol=1e-11 * max(1.0, np.abs(want).max()))
    pool, pool_g = sim.vortices()   # the last file holds the state after the last solve
    last = output.read_snapshot2_file(files[-1])
    np.testing.assert_array_equal(last["rings"], pool)
    np.testing.assert_array_equal(last["gammas"], pool_g)
    assert np.abs(L.calc_impulse(last)[7:]).max() > 0    # the wake carries impulse
    text = open(load_path).read().splitlines()
    assert len(text) == steps + 1
    np.testing.assert_allclose([[float(x) for x in ln.split("\t")] for ln in text], rows, rtol=1e-5, atol=1e-12)
    tsv = str(tmp_path / "impulse.tsv")
    assert tools.main(["calc_impulse", "--input", str(out_dir), "--output", tsv]) == 0
    got = np.array([[float(x) for x in ln.split("\t")] for ln in open(tsv).read().splitlines()])
    want = np.array([L.calc_impulse(output.read_snapshot2_file(f)) for f in files])
    assert got.shape == (steps + 1, 10)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-12)
