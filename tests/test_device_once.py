"""Host test of the per-device once-guard that sets kernel attributes
(shared-memory limits, cluster permissions) once on every device a process
uses, instead of once per process."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_device_once_guard(tmp_path):
    exe = tmp_path / "device_once_test"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-pthread", "-I", os.path.join(ROOT, "uvlm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "device_once_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "device_once ok" in r.stdout
