"""pytest configuration: the ``gpu`` marker and import paths.

Tests marked ``gpu`` need a B200 and the built CUDA library; everything else
runs on the CPU (oracle known-answer tests, host logic, C-ABI symbol checks).
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
