"""The header-only C++ adapter (include/uvlm_b200.hpp): a C++ host written
against the reference's UVLM:: API, compiled with g++ against the C-ABI
library.  CPU: it compiles and links.  GPU: it runs and agrees with the
oracle (the program exits non-zero on any failed check)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    import pyoracle

    from uvlm_b200 import _capi

    lib_dir = os.path.dirname(_capi.ensure_built())
    orc_dir = os.path.dirname(pyoracle.build())
    exe = tmp_path / "adapter_parity"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "cpp", "adapter_parity.cpp"), "-L", lib_dir,
           "-luvlm_b200", "-L", orc_dir, "-loracle", f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{orc_dir}", "-o",
           str(exe)]
    subprocess.run(cmd, check=True)
    return exe


def test_cpp_adapter_compiles_and_links(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_cpp_adapter_matches_oracle(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.parametrize("fatal", [False, True])
def test_cpp_adapter_error_modes(tmp_path, fatal):
    """UVLM::Error by default; with UVLM_B200_FATAL_ON_ERROR the reference's LOG(FATAL) behaviour: the
    message on stderr, then abort."""
    from uvlm_b200 import _capi

    lib_dir = os.path.dirname(_capi.ensure_built())
    exe = tmp_path / "fatal_mode"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "fatal_mode.cpp"), "-L", lib_dir, "-luvlm_b200",
           f"-Wl,-rpath,{lib_dir}", "-o", str(exe)] + (["-DUVLM_B200_FATAL_ON_ERROR"] if fatal else [])
    subprocess.run(cmd, check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    if fatal:
        assert r.returncode == -6  # SIGABRT
        assert "Check failed: WriteStateRecord: invalid argument" in r.stderr
    else:
        assert r.returncode == 0 and r.stdout.startswith("caught 1: WriteStateRecord: invalid argument")
