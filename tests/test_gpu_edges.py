"""Edge cases of the CUDA path against the FP64 oracle (B200).

Empty inputs (no targets, sheets without rings), ragged strip shapes (column
counts that leave a short last chunk, row counts that leave a short last row
group), the smallest wing the reference accepts (1 x 2 rings) and a batch of
one case.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sheet(rng, num, rows, cols):
    i = np.arange(rows + 1)[:, None]
    j = np.arange(cols + 1)[None, :]
    pos = np.zeros((num, rows + 1, cols + 1, 3))
    for n in range(num):
        pos[n, ..., 0] = 0.25 * i + 0.01 * rng.standard_normal((rows + 1, cols + 1))
        pos[n, ..., 1] = 0.0625 * j + 0.01 * rng.standard_normal((rows + 1, cols + 1))
        pos[n, ..., 2] = 0.3 * n + 0.05 * np.sin(0.7 * i + 0.3 * j)
    return pos, rng.standard_normal((num, rows, cols))


def test_no_targets_and_no_rings():
    import uvlm_b200 as U

    rng = np.random.default_rng(0)
    pos, gamma = _sheet(rng, 1, 3, 4)
    for prec in ("fp64", "mixed"):
        out = U.InducedVelocity(np.zeros((0, 3)), pos, gamma, prec)
        assert out.shape == (0, 3)
        # a sheet with one node row has no rings: zero velocity everywhere
        v = U.InducedVelocity(rng.standard_normal((5, 3)), pos[:, :1], np.zeros((1, 0, 4)), prec)
        assert np.all(v == 0.0)


@pytest.mark.parametrize("shape", [(1, 7, 66), (2, 5, 129), (1, 130, 3), (1, 9, 64), (1, 9, 65)])
def test_ragged_strips_both_precisions(shape):
    import pyoracle as o

    import uvlm_b200 as U

    rng = np.random.default_rng(sum(shape))
    pos, gamma = _sheet(rng, *shape)
    targets = np.concatenate([rng.uniform(-0.5, 4.5, size=(300, 3)), pos.reshape(-1, 3)[::7]])
    ref = o.sheet_induced_velocity(pos, gamma, targets)
    scale = np.max(np.abs(ref))
    got64 = U.InducedVelocity(targets, pos, gamma, "fp64")
    assert np.max(np.abs(got64 - ref)) <= 1e-12 * scale
    got32 = U.InducedVelocity(targets, pos, gamma, "mixed")
    assert np.all(np.isfinite(got32))
    assert np.max(np.abs(got32 - ref)) <= 1e-5 * scale


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_smallest_wing_matches_oracle(precision):
    import pyoracle as o

    import uvlm_b200 as U

    dt, steps = 0.1, 12
    kin = dict(alpha=math.radians(4), plug_amp=0.1, plug_omega=1.3)
    sim = U.SimpleSimulator(precision=precision)
    m = U.Morphing().set_alpha(kin["alpha"]).set_plug(kin["plug_amp"], kin["plug_omega"])
    sim.AddWing(U.RectGenerator(), m, 1.0, 2.0, 1, 2)
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("RK2")
    rows = sim.Run(steps, dt)
    sim.close()
    ref = o.Simulator()
    ref.add_wing(1.0, 2.0, 1, 2, kin=o.kinematics(**kin))
    ref.set_forward_flight((-1.0, 0.0, 0.0))
    ref.set_advection("RK2")
    want = ref.run(steps, dt)
    tol = 1e-8 if precision == "fp64" else 1e-5
    assert np.max(np.abs(np.asarray(rows)[:, 1:] - want[:, 1:])) <= tol * np.max(np.abs(want[:, 1:]))


def test_batch_of_one_smallest_case():
    import pyoracle as o

    import uvlm_b200 as U
    from uvlm_b200.batch import BatchSimulator

    dt, steps = 0.1, 10
    sim = BatchSimulator(precision="fp64", max_steps=steps)
    sim.add_case(U.Morphing().set_alpha(math.radians(4)).set_plug(0.1, 1.3), 1.0, 2.0, 1, 2, dt)
    sim.run(steps)
    L = sim.loads()
    sim.close()
    ref = o.Simulator()
    ref.add_wing(1.0, 2.0, 1, 2, kin=o.kinematics(alpha=math.radians(4), plug_amp=0.1, plug_omega=1.3))
    ref.set_forward_flight((-1.0, 0.0, 0.0))
    ref.set_advection("euler")
    want = ref.run(steps - 1, dt)
    assert np.max(np.abs(L[:, 0, 1:] - want[:, 1:])) <= 1e-9 * np.max(np.abs(want[:, 1:]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_velocity_at_points_of_the_current_state(precision):
    """SimpleSimulator::Velocity on a grid of points (the velocity-field
    tools' use) equals -ff + the oracle's induced velocity of the state."""
    import pyoracle as o

    import uvlm_b200 as U

    sim = U.SimpleSimulator(precision=precision)
    sim.AddWing(U.RectGenerator(), U.Morphing().set_alpha(0.08).set_plug(0.1, 1.0), 1.0, 4.0, 4, 8)
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("RK2")
    sim.Run(15, 0.15)
    st = sim.state()
    g = np.stack(np.meshgrid(np.linspace(-0.5, 3.5, 9), np.linspace(-2.5, 2.5, 7), [-0.3, 0.21], indexing="ij"),
                 -1).reshape(-1, 3)
    got = sim.Velocity(g)
    sim.close()
    ref = (o.sheet_induced_velocity(st["wing_pos"], st["wing_gamma"], g)
           + o.sheet_induced_velocity(st["wake_pos"], st["wake_gamma"], g) + np.array([1.0, 0.0, 0.0]))
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
