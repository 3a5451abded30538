"""Host-side checks of the C-ABI library (no GPU needed).

The library must load, export every function that include/uvlm_b200.h
declares, agree with the ctypes structure layouts, and refuse to create a
context loudly (UVLM_ERR_CUDA) when no CUDA device is present.
"""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "uvlm_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(uvlm_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_api():
    names = declared_functions()
    for must in ("uvlm_create", "uvlm_step", "uvlm_advection_advect", "uvlm_sheet_induced_velocity",
                 "uvlm_rings_solve_linear_problem", "uvlm_dense_solve"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from uvlm_b200 import _capi

    L = C.CDLL(_capi.ensure_built())
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # and the ctypes signature table covers the same set
    assert sorted(n for n, _, _ in _capi.SIGNATURES) == declared_functions()


def test_struct_layouts_match_header(tmp_path):
    from uvlm_b200 import _capi

    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "uvlm_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(uvlm_config), sizeof(uvlm_kinematics), sizeof(uvlm_wing_desc),
         sizeof(uvlm_step_stats));
  printf("%zu %zu %zu\n", offsetof(uvlm_config, gmres_tol), offsetof(uvlm_kinematics, origin),
         offsetof(uvlm_step_stats, stage_ms));
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(uvlm_batch_case), sizeof(uvlm_batch_config),
         offsetof(uvlm_batch_case, kin), offsetof(uvlm_batch_case, chebyshev_span),
         offsetof(uvlm_batch_config, max_steps), offsetof(uvlm_config, preconditioner));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    sizes = list(map(int, out))
    assert sizes[:4] == [C.sizeof(_capi.Config), C.sizeof(_capi.Kinematics), C.sizeof(_capi.WingDesc),
                         C.sizeof(_capi.StepStats)]
    assert sizes[4] == _capi.Config.gmres_tol.offset
    assert sizes[5] == _capi.Kinematics.origin.offset
    assert sizes[6] == _capi.StepStats.stage_ms.offset
    assert sizes[7:] == [C.sizeof(_capi.BatchCase), C.sizeof(_capi.BatchConfig), _capi.BatchCase.kin.offset,
                         _capi.BatchCase.chebyshev_span.offset, _capi.BatchConfig.max_steps.offset,
                         _capi.Config.preconditioner.offset]


def test_oracle_kinematics_layout_matches_product():
    import pyoracle
    from uvlm_b200 import _capi

    assert C.sizeof(pyoracle.Kinematics) == C.sizeof(_capi.Kinematics)
    assert [f[0] for f in pyoracle.Kinematics._fields_] == [f[0] for f in _capi.Kinematics._fields_]


def test_status_strings():
    from uvlm_b200 import _capi

    L = _capi.lib()
    assert L.uvlm_status_string(0) == b"ok"
    assert L.uvlm_status_string(3) == b"singular matrix"


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_create_without_device_fails_loudly():
    import uvlm_b200 as U

    with pytest.raises(U.UVLMError) as ei:
        U.SimpleSimulator()
    assert ei.value.code == 2


def test_invalid_advection_name_is_rejected_without_device():
    import uvlm_b200 as U

    with pytest.raises(U.UVLMError) as ei:
        U.AdvectFactory("RK3")
    assert ei.value.code == 1
    assert "euler" in str(ei.value)


@pytest.mark.parametrize("field,value,message", [
    ("precision", 7, "unknown precision"),
    ("advection", 4, "invalid configuration"),
    ("max_wake_rows", 0, "invalid configuration"),
    ("gmres_tol", 0.0, "invalid configuration"),
    ("preconditioner", 2, "invalid configuration"),
    ("nbody_fp64_stages", 8, "invalid configuration"),
    ("nbody_near_fp64", -1, "invalid configuration"),
    ("lu_pivoting", 2, "invalid configuration"),
    ("gmres_refresh_iter", -1, "invalid configuration"),
])
def test_invalid_configuration_is_rejected_before_the_device(field, value, message):
    """uvlm_create checks the configuration before it looks for a device, so a
    bad field reads UVLM_ERR_INVALID on any machine (and no context is made)."""
    from uvlm_b200 import _capi

    L = _capi.lib()
    cfg = _capi.Config()
    L.uvlm_config_default(C.byref(cfg))
    setattr(cfg, field, value)
    out = C.c_void_p(1)
    assert L.uvlm_create(C.byref(cfg), C.byref(out)) == 1
    assert out.value is None
    assert message in L.uvlm_global_last_error().decode()


def test_oracle_is_not_linked_into_the_product():
    from uvlm_b200 import _capi

    out = subprocess.run(["ldd", _capi.ensure_built()], capture_output=True, text=True).stdout
    assert "oracle" not in out
    syms = subprocess.run(["nm", "-D", "--defined-only", _capi.ensure_built()], capture_output=True,
                          text=True).stdout
    assert "orc_" not in syms
