"""Train the learned warm start for a single-wing workload.

    python -m uvlm_b200.train_warmstart --out uvlm_b200/weights/warmstart_heave_pitch_32x128.npz
    python -m uvlm_b200.train_warmstart --workload morphing --out uvlm_b200/weights/warmstart_morphing_24x96.npz

Training pairs come from the plain FP64 solver (fresh FP64 LU every step) on
seeded variations of the workload's kinematics:
  heave_pitch  32 x 128 rings, AR 8, heave 0.2 c sin(wt), pitch 10 deg
               sin(wt + 90 deg), k = 0.5, RK2; heave and pitch amplitudes
               within +-20 %, phase within +-0.3 rad;
  morphing     24 x 96 rings, AR 8, camber 0.05 sin(wt) x(1-x) and span bend
               0.1 sin(wt) y^2, k = 0.3, Euler; both amplitudes within
               +-20 %, phase within +-0.3 rad.
Each run
advances `--steps` steps with the wake held at `--wake-rows` rows; a random
`--sample` fraction of the panel pairs of every run is kept.  The network is
trained with the library's own forward/backward/Adam kernels.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import Morphing, RectGenerator, SimpleSimulator
from .warmstart import MLP


def make_sim(heave, pitch_deg, phase, wake_rows, rows=32, cols=128, span=8.0, omega=1.0):
    sim = SimpleSimulator(precision="fp64", erase_wake_after=wake_rows, max_wake_rows=wake_rows + 8)
    m = Morphing().set_plug(heave, omega).set_twist(math.radians(pitch_deg), omega, math.pi / 2 + phase)
    sim.AddWing(RectGenerator(), m, 1.0, span, rows, cols, (0.0, 0.0, 0.0))
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("RK2")
    return sim


def make_morphing_sim(cx, cy, phase, wake_rows, rows=24, cols=96, span=8.0, omega=0.6):
    sim = SimpleSimulator(precision="fp64", erase_wake_after=wake_rows, max_wake_rows=wake_rows + 8)
    m = Morphing().set_bend(cx, cy, omega, phase)
    sim.AddWing(RectGenerator(), m, 1.0, span, rows, cols, (0.0, 0.0, 0.0))
    sim.set_forward_flight([-1.0, 0.0, 0.0])
    sim.set_advection("euler")
    return sim


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--workload", default="heave_pitch", choices=["heave_pitch", "morphing"])
    ap.add_argument("--runs", type=int, default=50)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--wake-rows", type=int, default=100)
    ap.add_argument("--sample", type=float, default=0.1)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    rng = np.random.default_rng(a.seed)
    dt = 2 * math.pi / 40 if a.workload == "heave_pitch" else 2 * math.pi / 0.6 / 40
    Xs, Ts = [], []
    t0 = time.time()
    for r in range(a.runs):
        amp1 = 1 + 0.2 * rng.uniform(-1, 1)
        amp2 = 1 + 0.2 * rng.uniform(-1, 1)
        phase = 0.3 * rng.uniform(-1, 1)
        if a.workload == "heave_pitch":
            sim = make_sim(0.2 * amp1, 10.0 * amp2, phase, a.wake_rows)
            panels = 32 * 128
        else:
            sim = make_morphing_sim(0.05 * amp1, 0.1 * amp2, phase, a.wake_rows)
            panels = 24 * 96
        sim.begin()
        sim.collect_training_data(True, panels * (a.steps + 1))
        for s in range(a.steps + 1):
            sim.step(s, dt)
        X, T = sim.training_data()
        keep = rng.random(X.shape[0]) < a.sample
        Xs.append(X[keep])
        Ts.append(T[keep])
        sim.close()
        print(f"run {r}: {X.shape[0]} pairs, kept {int(keep.sum())}, {time.time() - t0:.0f} s", flush=True)
    X = np.concatenate(Xs)
    T = np.concatenate(Ts)
    net = MLP(seed=a.seed)
    net.fit_normalization(X, T)
    _, loss0 = net.gradients(X[:65536], T[:65536])
    loss = net.train(X, T, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed)
    net.save(a.out)
    meta = dict(workload=a.workload, runs=a.runs, steps=a.steps, solver_steps=a.runs * (a.steps + 1), wake_rows=a.wake_rows,
                samples=int(X.shape[0]), loss_before=loss0, loss_after=loss, epochs=a.epochs,
                seconds=time.time() - t0)
    with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
