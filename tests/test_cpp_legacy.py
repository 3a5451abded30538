"""The legacy AoS C++ API of the header-only adapter (include/uvlm_b200.hpp):
tests/cpp/legacy_parity.cpp mirrors the reference's own container, wing
builder, shed and linear tests, checks the container loads against the
oracle, and prints the load rows of simulator::Start, which are compared
with the oracle's restatement of the legacy loop (oracle/legacy_oracle.py).
CPU: it builds and its host-only checks pass.  GPU: everything else."""
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    import pyoracle

    from uvlm_b200 import _capi

    lib_dir = os.path.dirname(_capi.ensure_built())
    orc_dir = os.path.dirname(pyoracle.build())
    exe = tmp_path / "legacy_parity"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "cpp", "legacy_parity.cpp"), "-L", lib_dir,
           "-luvlm_b200", "-L", orc_dir, "-loracle", f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{orc_dir}", "-o",
           str(exe)]
    subprocess.run(cmd, check=True)
    return exe


def test_cpp_legacy_host_checks(tmp_path):
    r = subprocess.run([str(_build(tmp_path)), "cpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_legacy_gpu_checks(tmp_path):
    r = subprocess.run([str(_build(tmp_path)), "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["start", "start_joukowski"])
def test_cpp_legacy_start_matches_oracle(tmp_path, mode):
    import legacy_oracle as L
    import pyoracle as o

    from uvlm_b200 import output, tools

    out_dir = tmp_path / "result"
    out_dir.mkdir()
    r = subprocess.run([str(_build(tmp_path)), mode, str(out_dir)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.array([[float(x) for x in line.split()] for line in r.stdout.strip().splitlines()])
    X, Y = np.meshgrid(np.arange(4) / 3.0, np.arange(5) / 2.0, indexing="ij")
    pts = np.stack([X, Y, 0 * X], -1)
    wings, kins = [], []
    for w in range(2):
        wings.append(dict(rows=3, cols=4, points=pts, origin=(0.0, 0.0, 0.8 * w), chord=1.0, span=2.0))
        k = o.Kinematics()
        k.alpha, k.plug_amp, k.plug_omega, k.plug_phase = 0.08, 0.1, 1.0, 0.5 * w
        k.twist_amp, k.twist_omega, k.twist_phase = 0.05, 1.0, 0.3
        k.origin[2] = 0.8 * w
        kins.append(k)
    snaps = []
    ref = L.start(wings, kins, [1.0, 0.0, 0.0], 10, 2 * math.pi / 40, use_joukowski=mode == "start_joukowski",
                  snapshots=snaps)
    assert got.shape == ref.shape == (11, 11)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-8 * np.max(np.abs(ref[:, 1:])))
    # OutputSnapshot2 (simulator.cpp:118-160): one file per step
    files = tools.glob_result(str(out_dir))
    assert len(files) == 11
    for f, s in zip(files, snaps):
        d = output.read_snapshot2_file(f)
        assert d["t"] == s["t"] and [c["id"] for c in d["container_shapes"]] == [0, 1]
        np.testing.assert_allclose(d["rings"], s["rings"], rtol=0, atol=1e-10 * np.abs(s["rings"]).max())
        np.testing.assert_array_equal(d["rings0"], s["rings0"])
        np.testing.assert_allclose(d["gammas"], s["gammas"], rtol=0, atol=1e-8 * np.abs(s["gammas"]).max())
        np.testing.assert_allclose(d["mv_nodes"], s["mv_nodes"], rtol=0, atol=1e-8)
        np.testing.assert_allclose(d["mv_center"], s["mv_center"], rtol=0, atol=1e-8)
