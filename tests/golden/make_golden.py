"""Generates the golden fixtures of tests/golden/ with the CPU oracle.

    python tests/golden/make_golden.py

The reference itself cannot be compiled in this environment (Eigen3,
protobuf, glog, gflags, boost and its multiple_sheet submodule are absent), so
the fixtures come from the oracle, whose arithmetic is pinned by the
reference's own known-answer tests (tests/test_oracle_kats.py).  Each fixture
stores the load rows (t, CD, CL per wing) of every step and the final state.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

from cases import CASES, run_oracle  # noqa: E402


def main(names=None):
    for name, case in CASES.items():
        if names and name not in names:
            continue
        loads, st = run_oracle(case)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, loads=loads, wing_gamma=st["wing_gamma"], wake_gamma=st["wake_gamma"],
                            wake_pos=st["wake_pos"], wing_pos=st["wing_pos"])
        print(f"{name}: {loads.shape[0]} steps, final CL {loads[-1, 2]:.6f} -> {os.path.relpath(path, ROOT)}")


if __name__ == "__main__":
    main(sys.argv[1:])
