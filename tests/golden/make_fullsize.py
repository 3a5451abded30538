"""Generates the full-size fixtures of tests/golden/ with the CPU oracle.

    python tests/golden/make_fullsize.py [name ...]

The benchmark workloads at their full lattice sizes (32 x 128 heave/pitch,
4 x 16 x 64 tandem/biplane, 24 x 96 morphing), run by the FP64 oracle from
step 0 over the window given in cases.FULLSIZE.  The FullPivLU runs on all
host threads (bit-identical to the single-threaded elimination).  Each fixture
holds the load row of every step, the circulations every 10 steps and the
final wing circulations and wake nodes.  Takes tens of minutes on 8 cores.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

from cases import FULLSIZE  # noqa: E402


def run(case, threads):
    import pyoracle as o

    sim = o.Simulator()
    for w in case["wings"]:
        sim.add_wing(w["chord"], w["span"], w["rows"], w["cols"], origin=w["origin"], kin=o.kinematics(**w["kin"]))
    sim.set_forward_flight(case["ff"])
    sim.set_advection(case["advection"])
    sim.set_threads(threads)
    sim.set_lu_threads(threads)
    sim.begin()
    loads, gammas, steps_kept = [], [], []
    for s in range(case["steps"]):
        loads.append(sim.step(s, case["dt"]))
        if s % 10 == 9 or s == case["steps"] - 1:
            gammas.append(sim.state()["wing_gamma"])
            steps_kept.append(s)
        print(f"  step {s}: CL {loads[-1][2]:.9f}", flush=True)
    st = sim.state()
    return dict(loads=np.array(loads), gamma_steps=np.array(steps_kept), gammas=np.array(gammas),
                wing_gamma=st["wing_gamma"], wake_pos=st["wake_pos"], wake_gamma=st["wake_gamma"])


def main(names=None):
    threads = len(os.sched_getaffinity(0))
    for name, case in FULLSIZE.items():
        if names and name not in names:
            continue
        t0 = time.time()
        out = run(case, threads)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {case['steps']} steps in {time.time() - t0:.0f} s -> {os.path.relpath(path, ROOT)}", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
