"""Batched independent cases (uvlm_batch_*) against the FP64 oracle and the
single-case library path, on a B200.

Cases come from the seeded flapping-wing sweep (rows 4-16, even cols 8-64,
aspect ratio 2-10, k 0.1-1, heave 0.05-0.3, pitch 0-20 deg), cut to sizes the
oracle finishes in seconds.  Each case of the batch must reproduce its own
SimpleSimulator run: FP64 batch within 1e-9 of the oracle on the loads and
circulation; the mixed batch (FP32 N-body, FP32 LU + FP64 refinement) within
1e-6 relative.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 20


def _small_cases(n, seed=3):
    from uvlm_b200.batch import draw_cases

    cs = draw_cases(n, seed)
    for d in cs:  # cut to oracle-sized lattices, keep the drawn kinematics
        d["rows"] = 2 + d["rows"] // 4
        d["cols"] = 2 * (2 + d["cols"] // 16)
        d["span"] = min(d["span"], 6.0)
    return cs


def _oracle(d, steps, advection="euler"):
    import pyoracle as o

    sim = o.Simulator()
    kin = o.kinematics(plug_amp=d["heave"], plug_omega=d["omega"], twist_amp=math.radians(d["pitch_deg"]),
                       twist_omega=d["omega"], twist_phase=math.pi / 2)
    sim.add_wing(d["chord"], d["span"], d["rows"], d["cols"], kin=kin)
    sim.set_forward_flight((-1.0, 0.0, 0.0))
    sim.set_advection(advection)
    loads = sim.run(steps - 1, d["dt"])
    return np.asarray(loads), sim.state()


@pytest.mark.parametrize("advection", ["euler", "RK2"])
def test_batch_fp64_matches_oracle(advection):
    from uvlm_b200.batch import make_batch

    cases = _small_cases(5)
    sim = make_batch(cases, precision="fp64", advection=advection, max_steps=STEPS)
    sim.run(STEPS)
    L = sim.loads()
    assert L.shape == (STEPS, len(cases), 3)
    for c, d in enumerate(cases):
        ref, st = _oracle(d, STEPS, advection)
        np.testing.assert_allclose(L[:, c, 0], ref[:, 0], rtol=0, atol=1e-12)
        scale = np.max(np.abs(ref[:, 1:])) + 1e-30
        np.testing.assert_allclose(L[:, c, 1:], ref[:, 1:], rtol=0, atol=1e-9 * scale)
        got = sim.case_state(c)
        np.testing.assert_allclose(got["wing_gamma"], st["wing_gamma"][0], rtol=0,
                                   atol=1e-9 * np.max(np.abs(st["wing_gamma"])))
        np.testing.assert_allclose(got["wake_pos"], st["wake_pos"][0], rtol=0, atol=1e-9)
        np.testing.assert_allclose(got["wake_gamma"], st["wake_gamma"][0], rtol=0,
                                   atol=1e-9 * np.max(np.abs(st["wing_gamma"])))
    sim.close()


def test_batch_mixed_refinement_matches_oracle():
    from uvlm_b200.batch import make_batch

    cases = _small_cases(6, seed=11)
    sim = make_batch(cases, precision="mixed", max_steps=STEPS)
    sim.run(STEPS)
    L = sim.loads()
    sweeps, res = sim.solve_stats()
    assert np.all(res <= 1e-12)
    for c, d in enumerate(cases):
        ref, st = _oracle(d, STEPS)
        scale = np.max(np.abs(ref[:, 1:]))
        assert np.max(np.abs(L[:, c, 1:] - ref[:, 1:])) <= 1e-6 * scale
    sim.close()


def test_batch_graph_replay_equals_direct_launches():
    from uvlm_b200.batch import make_batch

    cases = _small_cases(7, seed=5)
    out = []
    for g in (True, False):
        # one pinned tile for both (each batch's autotuner could pick another)
        sim = make_batch(cases, precision="mixed", max_steps=12, use_graph=g, nbody_tile=0)
        sim.run(5)
        sim.run(7)
        out.append((sim.loads(), [sim.case_state(c)["wake_pos"] for c in range(len(cases))]))
        if g:
            assert sim.launches_per_step() > 10
        sim.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    for a, b in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(a, b)


def test_batch_case_equals_single_case_library_path():
    """A case inside a ragged batch gives the single-case FP64 path's answer."""
    import uvlm_b200 as U
    from uvlm_b200.batch import case_morphing, make_batch

    cases = _small_cases(4, seed=9)
    sim = make_batch(cases, precision="fp64", max_steps=10)
    sim.run(10)
    L = sim.loads()
    for c, d in enumerate(cases):
        one = U.SimpleSimulator(precision="fp64")
        one.AddWing(U.RectGenerator(), case_morphing(d), d["chord"], d["span"], d["rows"], d["cols"])
        one.set_forward_flight([-1.0, 0.0, 0.0])
        one.set_advection("euler")
        one.begin()
        rows = np.array([one.step(s, d["dt"]) for s in range(10)])
        np.testing.assert_allclose(L[:, c, 1:], rows[:, 1:], rtol=0, atol=1e-10 * np.max(np.abs(rows[:, 1:])))
        one.close()
    sim.close()


def test_batch_full_sweep_shapes_run():
    """The 256-case sweep at its drawn sizes: a few steps, finite loads,
    refinement converged in every case."""
    from uvlm_b200.batch import draw_cases, make_batch

    cases = draw_cases(256, seed=0)
    sim = make_batch(cases, precision="mixed", max_steps=8)
    sim.run(8)
    L = sim.loads()
    assert np.all(np.isfinite(L))
    sweeps, res = sim.solve_stats()
    assert np.all(res <= 1e-12)
    sim.close()


def test_batch_rejects_bad_cases():
    import uvlm_b200 as U
    from uvlm_b200.batch import BatchError, BatchSimulator

    sim = BatchSimulator()
    sim.add_case(U.Morphing(), 1.0, 4.0, 4, 7, 0.1)  # odd cols
    with pytest.raises(BatchError):
        sim.begin()
    sim2 = BatchSimulator(max_steps=3)
    sim2.add_case(U.Morphing(), 1.0, 4.0, 4, 8, 0.1)
    sim2.run(3)
    with pytest.raises(BatchError):
        sim2.run(1)
    sim2.close()


def test_batch_wide_and_narrow_cases_mixed_vs_oracle():
    """Cases wide enough for the padded packed walker (cols >= 48) and narrow
    ones in one mixed batch, each against its own oracle run."""
    from uvlm_b200.batch import make_batch

    rng = np.random.default_rng(21)
    cases = []
    for cols in (64, 8, 50, 12, 48):
        k = float(rng.uniform(0.3, 0.8))
        cases.append(dict(rows=3, cols=cols, chord=1.0, span=float(rng.uniform(3, 8)), k=k, omega=2 * k,
                          heave=float(rng.uniform(0.05, 0.2)), pitch_deg=float(rng.uniform(2, 15)),
                          dt=2 * math.pi / (2 * k) / 40))
    steps = 12
    sim = make_batch(cases, precision="mixed", max_steps=steps)
    sim.run(steps)
    L = sim.loads()
    sim.close()
    for c, d in enumerate(cases):
        ref, _ = _oracle(d, steps)
        scale = np.max(np.abs(ref[:, 1:]))
        assert np.max(np.abs(L[:, c, 1:] - ref[:, 1:])) <= 1e-6 * scale, d["cols"]


def test_batch_stale_factors_same_answer_fewer_factorizations():
    """Refining from the previous circulation with an earlier step's FP32
    factors converges to the same 1e-12 residual as a fresh factorisation
    every step, with fewer factorisations."""
    from uvlm_b200.batch import make_batch

    cases = _small_cases(6, seed=17)
    steps = 20
    out = {}
    for stale in (False, True):
        # one pinned tile for both: each batch's autotuner could pick another, and
        # another tile's FP32 rounding, grown by the wake over 20 steps, exceeds 1e-9
        sim = make_batch(cases, precision="mixed", max_steps=steps, stale_factors=stale, nbody_tile=0)
        sim.run(steps)
        out[stale] = (sim.loads(), sim.factorizations(), sim.solve_stats()[1])
        sim.close()
    assert out[False][1] == len(cases) * steps
    assert out[True][1] < out[False][1]
    assert np.all(out[True][2] <= 1e-12)
    scale = np.max(np.abs(out[False][0][:, :, 1:]))
    assert np.max(np.abs(out[True][0][:, :, 1:] - out[False][0][:, :, 1:])) <= 1e-9 * scale


def test_batch_tile_autotuner_is_fixed_under_graph_replay():
    """The tile autotuner picks one compiled FP32 tile at creation; every
    graph-replayed step runs it: the autotuned batch equals, bit for bit, a
    batch pinned to the tile it chose, with and without graph replay."""
    from uvlm_b200.batch import draw_cases, make_batch

    cases = draw_cases(12, seed=4)
    auto = make_batch(cases, precision="mixed", max_steps=30)
    name = auto.nbody_tile()
    assert name.startswith("fp32_") and name.endswith("_x2f"), name
    auto.run(20)
    tiles = ["fp32_h3_t2_b128_x2f", "fp32_h2_t2_b128_x2f", "fp32_h4_t2_b128_x2f"]
    outs = []
    for graph in (True, False):
        from uvlm_b200.batch import BatchSimulator, case_morphing

        sim = BatchSimulator(precision="mixed", max_steps=30, use_graph=graph, nbody_tile=tiles.index(name))
        for d in cases:
            sim.add_case(case_morphing(d), d["chord"], d["span"], d["rows"], d["cols"], d["dt"])
        assert sim.nbody_tile() == name
        sim.run(20)
        outs.append(sim.loads())
        sim.close()
    np.testing.assert_array_equal(auto.loads(), outs[0])
    np.testing.assert_array_equal(outs[0], outs[1])
    auto.close()


def test_every_batch_tile_agrees_with_the_fp64_batch():
    from uvlm_b200.batch import BatchSimulator, case_morphing, draw_cases

    cases = draw_cases(6, seed=9)

    def run(precision, tile=-1):
        sim = BatchSimulator(precision=precision, max_steps=16, nbody_tile=tile)
        for d in cases:
            sim.add_case(case_morphing(d), d["chord"], d["span"], d["rows"], d["cols"], d["dt"])
        sim.run(15)
        out = sim.loads()
        sim.close()
        return out

    ref = run("fp64")
    scale = np.max(np.abs(ref[:, :, 1:]))
    for t in range(3):
        got = run("mixed", t)
        assert np.max(np.abs(got[:, :, 1:] - ref[:, :, 1:])) <= 1e-6 * scale, t
