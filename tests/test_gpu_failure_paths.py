"""Failure paths of the accelerated solve, driven from the host (needs a B200).

* The GMRES iteration cap: with gmres_max_iter = 1 the stale-LU GMRES stops
  early and the plain fresh-LU solve (an FP64 LU of the step's FP64 matrix)
  gives the circulation; with every N-body stage in FP64 the result is the
  plain FP64 form's to rounding.
* A non-finite learned guess (NaN weights set from the host) takes the same
  fallback and the step still succeeds.
* A bounded device wait that runs out (a flag nothing sets, a short limit)
  returns UVLM_ERR_TIMEOUT, and the device stays usable.
No kernel is made to fault: every failure comes from host-side inputs or a
wait limit, and every wait in the library gives up after its limit.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import CASES, make_gpu_sim  # noqa: E402

pytestmark = pytest.mark.gpu

ALL_FP64 = ("rhs", "loads", "advect")


def _run(case, steps, sim):
    sim.begin()
    rows, gammas, paths = [], [], []
    for s in range(steps):
        rows.append(sim.step(s, case["dt"]))
        gammas.append(sim.state()["wing_gamma"])
        paths.append(int(sim.stats().solve_path))
    return np.array(rows), np.array(gammas), paths


def test_gmres_cap_takes_the_plain_fresh_lu_solve():
    case = CASES["morph_camber_euler_4x8"]
    steps = case["steps"]
    _, g64, _ = _run(case, steps, make_gpu_sim(case))
    _, gmx, paths = _run(case, steps, make_gpu_sim(case, precision="mixed", solver="gmres_stale",
                                                   warm_start="previous", gmres_max_iter=1, fp64_stages=ALL_FP64))
    assert 2 in paths, paths
    err = np.max(np.abs(gmx - g64)) / np.max(np.abs(g64))
    print("solve paths", paths, "circulation vs plain FP64", err)
    assert err <= 1e-10


def test_nonfinite_learned_guess_takes_the_fallback():
    from uvlm_b200.warmstart import MLP

    case = CASES["rk2_heave_pitch_4x8"]
    steps = case["steps"]
    _, g64, _ = _run(case, steps, make_gpu_sim(case))
    net = MLP(seed=1)
    p = net.params()
    p[:] = np.nan
    net.set_params(p)
    sim = make_gpu_sim(case, precision="mixed", solver="gmres_stale", warm_start="mlp", fp64_stages=ALL_FP64)
    sim.set_mlp(net)
    _, gmx, paths = _run(case, steps, sim)
    # the guess is used from step 2 on; every such step falls back
    assert all(q == 2 for q in paths[2:]), paths
    assert np.all(np.isfinite(gmx))
    assert np.max(np.abs(gmx - g64)) / np.max(np.abs(g64)) <= 1e-10


def test_bounded_wait_times_out_and_the_device_stays_usable():
    import uvlm_b200 as U

    rc = U.lib().uvlm_check_bounded_wait(0, 20000)
    assert rc == 7  # UVLM_ERR_TIMEOUT
    assert "gave up" in U.lib().uvlm_global_last_error().decode()
    # the library and the device still work: a dense solve and a short run
    rng = np.random.default_rng(2)
    A = rng.standard_normal((300, 300)) + 30 * np.eye(300)
    b = rng.standard_normal(300)
    x, _ = U.dense_solve(A, b)
    assert np.max(np.abs(A @ x - b)) <= 1e-10 * np.max(np.abs(b))
    case = CASES["rk2_heave_pitch_4x8"]
    rows = make_gpu_sim(case).Run(4, case["dt"])
    assert np.all(np.isfinite(rows))


def test_wait_limit_setter_validates_and_restores():
    import uvlm_b200 as U

    assert U.lib().uvlm_set_wait_limit(0, -1) == 1
    assert U.lib().uvlm_set_wait_limit(0, 10 ** 8) == 0
    assert U.lib().uvlm_set_wait_limit(0, 0) == 0  # back to the default
