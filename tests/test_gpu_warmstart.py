"""Learned warm start: kernels vs autograd, training, and what it gains (B200).

The MLP's forward/backward/Adam are the library's own CUDA kernels.  Its
gradients are checked against PyTorch CPU FP64 autograd of the same network
(same BF16-rounded weights, exact-erf GELU).  The ablation trains the network
on pairs the plain FP64 solver produces for seeded heave/pitch kinematics and
compares, on held-out kinematics, the GMRES initial residual and iteration
count of the MLP guess against the linear extrapolation 2 G_n - G_{n-1}.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch_reference(net, X, T):
    import torch

    mean = torch.tensor(net.mean, dtype=torch.float64)
    std = torch.tensor(net.std, dtype=torch.float64)
    s = net.out_scale
    params = []
    h = (torch.tensor(X, dtype=torch.float64) - mean) / std
    for i, (W, b) in enumerate(net.layers()):
        Wt = torch.tensor(W).to(torch.bfloat16).to(torch.float64).requires_grad_(True)
        bt = torch.tensor(b, dtype=torch.float64).requires_grad_(True)
        params += [Wt, bt]
        z = h @ Wt + bt
        h = 0.5 * z * (1 + torch.erf(z / math.sqrt(2))) if i < 3 else z
    y = h[:, 0]
    loss = torch.mean((y - torch.tensor(T, dtype=torch.float64) / s) ** 2)
    loss.backward()
    grads = np.concatenate([np.concatenate([p.grad.numpy().ravel() for p in params[2 * i:2 * i + 2]])
                            for i in range(4)])
    return grads, float(loss.detach()), (y.detach().numpy() * s)


def test_mlp_forward_and_gradients_match_autograd():
    from uvlm_b200.warmstart import MLP

    rng = np.random.default_rng(5)
    net = MLP(seed=3)
    X = rng.standard_normal((96, 8)).astype(np.float32)
    T = (0.3 * rng.standard_normal(96)).astype(np.float32)
    net.set_normalization(rng.standard_normal(8) * 0.1, 0.5 + rng.random(8), 0.7)
    g_ref, loss_ref, y_ref = _torch_reference(net, X, T)
    y = net.forward(X)
    np.testing.assert_allclose(y, y_ref, rtol=1e-4, atol=1e-5 * np.max(np.abs(y_ref)))
    g, loss = net.gradients(X, T)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.max(np.abs(g - g_ref)) <= 1e-4 * np.max(np.abs(g_ref))


def _torch_forward_bf16_activations(net, X):
    """FP64 forward of the same network with the BF16 rounding the tensor cores see: BF16 weights of every
    layer, the hidden layers' inputs (the GELU outputs of layers 1 and 2) rounded to BF16, and GELU in the
    tanh form the tensor-core inference evaluates."""
    import torch

    h = (torch.tensor(X, dtype=torch.float64) - torch.tensor(net.mean, dtype=torch.float64)) / torch.tensor(
        net.std, dtype=torch.float64)
    for i, (W, b) in enumerate(net.layers()):
        if i in (1, 2):
            h = h.to(torch.float32).to(torch.bfloat16).to(torch.float64)
        z = h @ torch.tensor(W).to(torch.bfloat16).to(torch.float64) + torch.tensor(b, dtype=torch.float64)
        h = 0.5 * z * (1 + torch.tanh(math.sqrt(2 / math.pi) * (z + 0.044715 * z ** 3))) if i < 3 else z
    return h[:, 0].numpy() * net.out_scale


@pytest.mark.parametrize("n", [1, 128, 1000, 4096])
def test_mlp_tensor_core_inference_matches_fp64_reference(n):
    """The tcgen05 inference (BF16 activations, tanh-form GELU, FP32 accumulation in TMEM) against FP64
    autograd-free references: with the same BF16 roundings and GELU form to 2e-3 of max |y|, and against the
    FP32-activation network (the SIMT forward and FP64 with exact erf activations) to the BF16 activation
    level, 2e-2 of max |y|."""
    import os

    from uvlm_b200.warmstart import MLP

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    net = MLP.load(os.path.join(root, "uvlm_b200", "weights", "warmstart_heave_pitch_32x128.npz"))
    rng = np.random.default_rng(n)
    X = (net.mean + net.std * rng.standard_normal((n, 8))).astype(np.float32)
    y_tc = net.forward_tc(X)
    y_simt = net.forward(X)
    y_bf = _torch_forward_bf16_activations(net, X)
    _, _, y_fp = _torch_reference(net, X, np.zeros(n, np.float32))
    scale = max(np.max(np.abs(y_fp)), 1e-30)
    assert np.all(np.isfinite(y_tc))
    assert np.max(np.abs(y_tc - y_bf)) <= 2e-3 * scale
    assert np.max(np.abs(y_tc - y_fp)) <= 2e-2 * scale
    assert np.max(np.abs(y_tc - y_simt)) <= 2e-2 * scale


def test_mlp_training_fits_a_smooth_target():
    from uvlm_b200.warmstart import MLP

    rng = np.random.default_rng(8)
    X = rng.standard_normal((20000, 8)).astype(np.float32)
    T = (np.tanh(X[:, 0] - 0.5 * X[:, 3]) * 0.2 + 0.05 * X[:, 6] * X[:, 7]).astype(np.float32)
    net = MLP(seed=1)
    net.fit_normalization(X, T)
    _, loss0 = net.gradients(X[:4096], T[:4096])
    loss = net.train(X, T, epochs=15, batch=1024, lr=2e-3)
    assert loss < 0.02 * loss0


def _heave_pitch_sim(U, precision, heave, pitch_deg, phase, warm="previous"):
    sim = U.SimpleSimulator(precision=precision, warm_start=warm)
    m = U.Morphing().set_plug(heave, 1.0).set_twist(math.radians(pitch_deg), 1.0, math.pi / 2 + phase)
    sim.AddWing(U.RectGenerator(), m, 1.0, 4.0, 4, 8)
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("RK2")
    return sim


def test_learned_warm_start_gain_over_extrapolation():
    import uvlm_b200 as U
    from uvlm_b200.warmstart import MLP, collect

    dt, steps = 2 * math.pi / 40, 80
    rng = np.random.default_rng(0)
    variants = [(0.2 * (0.8 + 0.4 * rng.random()), 10 * (0.8 + 0.4 * rng.random()), 0.3 * rng.standard_normal())
                for _ in range(6)]
    X, T = collect(lambda v: _heave_pitch_sim(U, "fp64", *v), variants, steps, dt)
    assert X.shape[0] == 6 * (steps - 1) * 32
    net = MLP(seed=0)
    net.fit_normalization(X, T)
    net.train(X, T, epochs=60, batch=512, lr=1e-3)

    held_out = (0.21, 11.0, 0.17)
    res = {}
    for warm in ("extrapolate", "mlp"):
        sim = _heave_pitch_sim(U, "mixed", *held_out, warm=warm)
        if warm == "mlp":
            sim.set_mlp(net)
        sim.begin()
        r0, its, rows = [], [], []
        for s in range(steps + 1):
            rows.append(sim.step(s, dt))
            st = sim.stats()
            if s >= 3:
                r0.append(st.initial_residual)
                its.append(st.gmres_iters)
        res[warm] = (float(np.mean(r0)), int(np.sum(its)), np.array(rows))
        sim.close()
    print(f"initial relative residual: extrapolation {res['extrapolate'][0]:.3e}, MLP {res['mlp'][0]:.3e}; "
          f"GMRES iterations: {res['extrapolate'][1]} vs {res['mlp'][1]}")
    # same converged answer either way
    np.testing.assert_allclose(res["mlp"][2], res["extrapolate"][2], rtol=0, atol=1e-9)
    # the network's guess starts closer than the extrapolation
    assert res["mlp"][0] < res["extrapolate"][0]


def test_shipped_weights_beat_extrapolation_on_the_workload():
    """The committed network (trained on 20k plain-solver steps of seeded
    heave/pitch variations, 32 x 128 rings) starts the GMRES solve of the
    workload itself closer than the extrapolation, and the converged answer is
    the same."""
    import os

    import uvlm_b200 as U
    from uvlm_b200.warmstart import MLP

    path = os.path.join(os.path.dirname(U.__file__), "weights", "warmstart_heave_pitch_32x128.npz")
    net = MLP.load(path)
    dt, steps = 2 * math.pi / 40, 40
    res = {}
    for warm in ("extrapolate", "mlp"):
        sim = U.SimpleSimulator(precision="mixed", warm_start=warm)
        if warm == "mlp":
            sim.set_mlp(net)
        m = U.Morphing().set_plug(0.2, 1.0).set_twist(math.radians(10), 1.0, math.pi / 2)
        sim.AddWing(U.RectGenerator(), m, 1.0, 8.0, 32, 128)
        sim.set_forward_flight([-1.0, 0.0, 0.0])
        sim.set_advection("RK2")
        sim.begin()
        r0, rows = [], []
        for s in range(steps + 1):
            rows.append(sim.step(s, dt))
            if s >= 3:
                r0.append(sim.stats().initial_residual)
        res[warm] = (float(np.mean(r0)), np.array(rows))
        sim.close()
    print(f"initial relative residual on the workload: extrapolation {res['extrapolate'][0]:.3e}, "
          f"MLP {res['mlp'][0]:.3e}")
    assert res["mlp"][0] < 0.5 * res["extrapolate"][0]
    # both converge to ||b - A g|| <= 1e-12 ||b||; the FP32 N-body carries
    # the remaining difference forward, so compare at the mixed form's 1e-6
    scale = np.max(np.abs(res["extrapolate"][1][:, 1:]))
    np.testing.assert_allclose(res["mlp"][1][:, 1:], res["extrapolate"][1][:, 1:], rtol=0, atol=1e-6 * scale)


def test_shipped_morphing_weights_beat_extrapolation():
    """The committed network for the morphing wing (24 x 96, camber and span
    bend, Euler; trained on 20k plain-solver steps of seeded variations)
    starts the GMRES solve closer than the extrapolation."""
    import os

    import uvlm_b200 as U
    from uvlm_b200.warmstart import MLP

    path = os.path.join(os.path.dirname(U.__file__), "weights", "warmstart_morphing_24x96.npz")
    net = MLP.load(path)
    dt, steps = 2 * math.pi / 0.6 / 40, 40
    res = {}
    for warm in ("extrapolate", "mlp"):
        sim = U.SimpleSimulator(precision="mixed", warm_start=warm)
        if warm == "mlp":
            sim.set_mlp(net)
        sim.AddWing(U.RectGenerator(), U.Morphing().set_bend(0.05, 0.1, 0.6), 1.0, 8.0, 24, 96)
        sim.set_forward_flight([-1.0, 0.0, 0.0])
        sim.set_advection("euler")
        sim.begin()
        r0, rows = [], []
        for s in range(steps + 1):
            rows.append(sim.step(s, dt))
            if s >= 3:
                r0.append(sim.stats().initial_residual)
        res[warm] = (float(np.mean(r0)), np.array(rows))
        sim.close()
    print(f"morphing: initial residual extrapolation {res['extrapolate'][0]:.3e}, MLP {res['mlp'][0]:.3e}")
    assert res["mlp"][0] < 0.5 * res["extrapolate"][0]
    scale = np.max(np.abs(res["extrapolate"][1][:, 1:]))
    np.testing.assert_allclose(res["mlp"][1][:, 1:], res["extrapolate"][1][:, 1:], rtol=0, atol=1e-6 * scale)
