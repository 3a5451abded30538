"""Properties at the benchmark's full size (B200): a 32 x 128 wing (4096 rings)
with a 400-row wake (51,200 rings), RK2, heave 0.2 sin(wt) + pitch
10 deg sin(wt + 90 deg), and the 4 x 16 x 64 tandem arrangement with 300 wake
rows per wing.

The oracle cannot run a whole step at this size in test time, so full-size
parity rests on properties that do not depend on the size:

* the N-body at a sample of targets (wake nodes, which see their own sheet's
  cut-offs, and wing collocation points) against the FP64 oracle;
* linearity of the N-body in the circulations (scaling by 2 is exact in
  every precision; sums agree to rounding);
* the dense solve at N = 4096: residual and agreement with LAPACK;
* one mixed-precision MainLoop against the plain FP64 MainLoop from the same
  full-size state (circulations, load row, advected wake).
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 2 * math.pi / 40
OMEGA = 1.0


def _move(x, y, t, z0=0.0, phase=0.0, heave=0.2, pitch=math.radians(10)):
    th = pitch * math.sin(OMEGA * t + phase + math.pi / 2)
    z = heave * math.sin(OMEGA * t + phase)
    return np.stack(np.broadcast_arrays(math.cos(th) * x, y, -math.sin(th) * x + z + z0), -1)


def _wing_and_wake(rows, cols, span, wake_rows, seed, x0=0.0, z0=0.0, phase=0.0, heave=0.2,
                   pitch=math.radians(10), dt=DT):
    """A moved rectangular lattice and its trailing edge convected at U = 1 for wake_rows rows, with a
    small seeded roll-up perturbation; smooth circulations."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0, 1.0, rows + 1)
    ys = np.linspace(-span / 2, span / 2, cols + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    t = wake_rows * dt
    wing = _move(X, Y, t, z0, phase, heave, pitch) + np.array([x0, 0.0, 0.0])
    wake = np.stack([_move(np.full(cols + 1, 1.0), ys, t - i * dt, z0, phase, heave, pitch)
                     + np.array([x0 + i * dt, 0.0, 0.0]) for i in range(wake_rows + 1)])
    wake[1:] += 0.003 * np.sqrt(np.arange(1, wake_rows + 1))[:, None, None] * rng.standard_normal(wake[1:].shape)
    g = 0.1 * np.sqrt(np.clip(1 - np.linspace(-1, 1, cols) ** 2, 0, None))
    wing_gamma = np.tile(g, (rows, 1)) * np.linspace(1, 0.2, rows)[:, None]
    wake_gamma = np.stack([g * 0.1 * math.sin(OMEGA * (t - i * dt) + phase) for i in range(wake_rows)])
    wake_gamma = wake_gamma + 1e-3 * rng.standard_normal(wake_gamma.shape)
    return wing, wing_gamma, wake, wake_gamma


def _heave_pitch():
    w, wg, k, kg = _wing_and_wake(32, 128, 8.0, 400, seed=1)
    return w[None], wg[None], k[None], kg[None]


def _tandem():
    parts = [_wing_and_wake(16, 64, 4.0, 300, seed=2 + q, x0=x, z0=z, phase=q * math.pi / 2, heave=0.15,
                            pitch=math.radians(15), dt=2 * math.pi / 0.8 / 40)
             for q, (x, z) in enumerate([(0.0, 0.0), (0.0, 0.5), (1.5, 0.0), (1.5, 0.5)])]
    return tuple(np.stack([p[i] for p in parts]) for i in range(4))


def _collocation(pos):
    return 0.25 * (pos[:, :-1, :-1] + pos[:, :-1, 1:] + pos[:, 1:, :-1] + pos[:, 1:, 1:])


def _targets(wing, wake):
    return np.concatenate([wake[:, 1:].reshape(-1, 3), _collocation(wing).reshape(-1, 3)])


def _velocity(M, x, wing, wg, wake, kg, precision):
    return (M.InducedVelocity(x, wing, wg, precision=precision)
            + M.InducedVelocity(x, wake, kg, precision=precision))


@pytest.mark.parametrize("case", ["heave_pitch", "tandem"])
def test_nbody_matches_oracle_on_sampled_targets(case):
    import pyoracle as o

    import uvlm_b200 as M

    wing, wg, wake, kg = _heave_pitch() if case == "heave_pitch" else _tandem()
    x = _targets(wing, wake)
    assert x.shape[0] == {"heave_pitch": 400 * 129 + 4096, "tandem": 4 * 300 * 65 + 4096}[case]
    v64 = _velocity(M, x, wing, wg, wake, kg, "fp64")
    v32 = _velocity(M, x, wing, wg, wake, kg, "mixed")
    rng = np.random.default_rng(7)
    n_wake = x.shape[0] - 4096
    pick = np.concatenate([rng.choice(n_wake, 40, replace=False), n_wake + rng.choice(4096, 24, replace=False),
                           [0, n_wake - 1, n_wake]])
    ref = o.sheet_induced_velocity(wing, wg, x[pick]) + o.sheet_induced_velocity(wake, kg, x[pick])
    scale = np.abs(ref).max()
    assert np.abs(v64[pick] - ref).max() <= 1e-12 * scale
    err = np.abs(v32[pick] - ref).max(axis=1)
    mag = np.linalg.norm(ref, axis=1)
    assert np.all(err <= 2e-5 * mag + 1e-6 * scale)
    # the FP32 form against the FP64 form at every target
    e_all = np.abs(v32 - v64).max(axis=1)
    assert np.all(e_all <= 2e-5 * np.linalg.norm(v64, axis=1) + 1e-6 * np.abs(v64).max())


def test_nbody_is_linear_in_the_circulations():
    import uvlm_b200 as M

    wing, wg, wake, kg = _heave_pitch()
    x = _targets(wing, wake)
    g2 = np.random.default_rng(3).standard_normal(kg.shape) * 0.01
    for precision in ("fp64", "mixed"):
        v = M.InducedVelocity(x, wake, kg, precision=precision)
        v2 = M.InducedVelocity(x, wake, 2.0 * kg, precision=precision)
        np.testing.assert_array_equal(v2, 2.0 * v)          # scaling by 2 is exact in FP32 and FP64
        vb = M.InducedVelocity(x, wake, g2, precision=precision)
        vs = M.InducedVelocity(x, wake, kg + g2, precision=precision)
        tol = (1e-13 if precision == "fp64" else 2e-6) * max(np.abs(v).max(), np.abs(vb).max())
        assert np.abs(vs - v - vb).max() <= tol


def test_dense_solve_at_4096():
    import uvlm_b200 as M

    n = 4096
    rng = np.random.default_rng(4)
    # influence-like: a dominant diagonal, a smooth rank-4 part and a random part of spectral radius about 1
    u = np.stack([np.cos((k + 1) * np.linspace(0, math.pi, n)) for k in range(4)], 1)
    A = rng.standard_normal((n, n)) / np.sqrt(n) + 0.5 * (u @ u.T) / n + np.diag(2.0 + rng.random(n))
    b = rng.standard_normal(n)
    ref = np.linalg.solve(A, b)
    for method in ("fp64", "tf32"):
        x, it = M.dense_solve(A, b, method)
        assert np.linalg.norm(b - A @ x) <= 1e-12 * np.linalg.norm(b)
        np.testing.assert_allclose(x, ref, rtol=0, atol=1e-11 * np.abs(ref).max())
        if method != "fp64":
            assert it <= 20


def _sim(M, precision):
    m = M.Morphing().set_plug(0.2, OMEGA).set_twist(math.radians(10), OMEGA, math.pi / 2)
    kw = dict(solver="gmres_stale", warm_start="extrapolate") if precision == "mixed" else {}
    sim = M.SimpleSimulator(precision=precision, erase_wake_after=400, max_wake_rows=408, **kw)
    sim.AddWing(M.RectGenerator(), m, 1.0, 8.0, 32, 128)
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("RK2")
    return sim


def test_mixed_mainloop_matches_fp64_from_a_full_size_state():
    import uvlm_b200 as M

    sims = {p: _sim(M, p) for p in ("fp64", "mixed")}
    wing, wg, wake, kg = _heave_pitch()
    rows, states = {}, {}
    for p, sim in sims.items():
        sim.begin()
        sim.step(0, DT)
        sim.set_state(400, wing, wake, wg, 0.99 * wg, kg)
        rows[p] = np.array([sim.step(s, DT) for s in range(401, 404)])
        states[p] = sim.state()
        sim.close()
    st64, st32 = states["fp64"], states["mixed"]
    assert st32["wake_gamma"].shape == st64["wake_gamma"].shape and st64["wake_gamma"].shape[1] >= 400
    g64 = st64["wing_gamma"]
    assert np.abs(st32["wing_gamma"] - g64).max() <= 1e-6 * np.abs(g64).max()
    kg64 = st64["wake_gamma"]
    assert np.abs(st32["wake_gamma"] - kg64).max() <= 1e-6 * np.abs(g64).max()
    # rows shed before the three steps are copies of the set state in both forms
    np.testing.assert_array_equal(st32["wake_gamma"][:, 3:], kg64[:, 3:])
    load = rows["fp64"][:, 1:]
    assert np.abs(rows["mixed"][:, 1:] - load).max() <= 1e-6 * np.abs(load).max()
    # FP32 velocities (error ~1e-6 of the induced velocity) moved through three RK2 steps of dt = 0.157
    assert np.abs(st32["wake_pos"] - st64["wake_pos"]).max() <= 1e-5
