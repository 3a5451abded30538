"""ctypes declarations of the C-ABI in include/uvlm_b200.h.

The shared library is built in-tree (uvlm_b200/libuvlm_b200.so).  Loading it
never falls back to anything else: if the library is missing and cannot be
built, or no CUDA device is present when a context is created, the call
raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libuvlm_b200.so")

UVLM_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "singular matrix", 4: "non-finite value",
          5: "call out of order", 6: "capacity exceeded", 7: "device wait timed out", 8: "unsupported"}

PRECISION = {"fp64": 0, "mixed": 1}
SOLVER = {"lu": 0, "gmres_stale": 1}
WARM = {"previous": 0, "extrapolate": 1, "mlp": 2}
LU_PREC = {"tf32": 0, "bf16": 1}
ADVECT = {"euler": 0, "RK2": 1, "RK4": 2, "AB2": 3}


class Config(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("solver", C.c_int32), ("warm_start", C.c_int32),
        ("lu_precision", C.c_int32), ("advection", C.c_int32), ("rk_ignore_rows", C.c_int32),
        ("max_wake_rows", C.c_int64), ("erase_wake_after", C.c_int64),
        ("gmres_restart", C.c_int32), ("gmres_max_iter", C.c_int32), ("gmres_tol", C.c_double),
        ("device", C.c_int32), ("compute_loads", C.c_int32), ("assembly_fp64", C.c_int32),
        ("nbody_variant", C.c_int32), ("preconditioner", C.c_int32), ("nbody_fp64_stages", C.c_int32),
        ("nbody_near_fp64", C.c_int32), ("lu_pivoting", C.c_int32), ("gmres_refresh_iter", C.c_int32),
    ]


class Kinematics(C.Structure):
    _fields_ = [
        ("alpha", C.c_double),
        ("plug_amp", C.c_double), ("plug_omega", C.c_double), ("plug_phase", C.c_double),
        ("flap_amp", C.c_double), ("flap_omega", C.c_double), ("flap_phase", C.c_double),
        ("twist_amp", C.c_double), ("twist_span_slope", C.c_double),
        ("twist_omega", C.c_double), ("twist_phase", C.c_double),
        ("bend_cx", C.c_double), ("bend_cy", C.c_double),
        ("bend_omega", C.c_double), ("bend_phase", C.c_double),
        ("origin", C.c_double * 3),
    ]


class WingDesc(C.Structure):
    _fields_ = [
        ("chord", C.c_double), ("span", C.c_double), ("rows", C.c_int64), ("cols", C.c_int64),
        ("origin", C.c_double * 3), ("chebyshev_chord", C.c_int32), ("chebyshev_span", C.c_int32),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("t", C.c_double), ("solve_path", C.c_int32), ("gmres_iters", C.c_int32),
        ("residual", C.c_double), ("refactored", C.c_int32), ("wake_rows", C.c_int32),
        ("stage_ms", C.c_double * 8), ("nbody_variant", C.c_int32), ("pad_", C.c_int32),
        ("initial_residual", C.c_double), ("nbody_ms", C.c_double), ("factor_ms", C.c_double),
        ("inverse_ms", C.c_double), ("stage_variant", C.c_int32 * 4),
    ]


class BatchCase(C.Structure):
    _fields_ = [
        ("chord", C.c_double), ("span", C.c_double), ("rows", C.c_int64), ("cols", C.c_int64),
        ("origin", C.c_double * 3), ("forward_flight", C.c_double * 3), ("dt", C.c_double),
        ("kin", Kinematics), ("chebyshev_chord", C.c_int32), ("chebyshev_span", C.c_int32),
    ]


class BatchConfig(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("advection", C.c_int32), ("rk_ignore_rows", C.c_int32),
        ("refine_max_iter", C.c_int32), ("refine_tol", C.c_double), ("max_steps", C.c_int64),
        ("device", C.c_int32), ("use_graph", C.c_int32), ("stale_factors", C.c_int32), ("nbody_tile", C.c_int32),
    ]


_P = C.POINTER(C.c_double)
_I = C.c_int64
_V = C.c_void_p

# (name, restype, argtypes): every symbol declared in include/uvlm_b200.h
SIGNATURES = [
    ("uvlm_config_default", None, [C.POINTER(Config)]),
    ("uvlm_create", C.c_int, [C.POINTER(Config), C.POINTER(_V)]),
    ("uvlm_destroy", C.c_int, [_V]),
    ("uvlm_last_error", C.c_char_p, [_V]),
    ("uvlm_global_last_error", C.c_char_p, []),
    ("uvlm_status_string", C.c_char_p, [C.c_int]),
    ("uvlm_add_wing", C.c_int, [_V, C.POINTER(WingDesc), C.POINTER(Kinematics)]),
    ("uvlm_add_wing_nodes", C.c_int, [_V, _I, _I, _P, C.c_double, C.c_double, _P, C.POINTER(Kinematics)]),
    ("uvlm_set_wait_limit", C.c_int, [C.c_int32, _I]),
    ("uvlm_check_bounded_wait", C.c_int, [C.c_int32, _I]),
    ("uvlm_set_forward_flight", C.c_int, [_V, _P]),
    ("uvlm_set_advection", C.c_int, [_V, C.c_char_p]),
    ("uvlm_begin", C.c_int, [_V]),
    ("uvlm_step", C.c_int, [_V, _I, C.c_double, _P]),
    ("uvlm_stage_kinematics", C.c_int, [_V, _I, C.c_double]),
    ("uvlm_stage_assemble", C.c_int, [_V]),
    ("uvlm_stage_rhs", C.c_int, [_V]),
    ("uvlm_stage_solve", C.c_int, [_V]),
    ("uvlm_stage_loads", C.c_int, [_V]),
    ("uvlm_stage_advect", C.c_int, [_V, _P]),
    ("uvlm_run", C.c_int, [_V, _I, C.c_double, _P]),
    ("uvlm_erase_oldest_wake", C.c_int, [_V]),
    ("uvlm_get_sizes", C.c_int, [_V, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]),
    ("uvlm_get_state", C.c_int, [_V, _P, _P, _P, _P, _P, _P]),
    ("uvlm_set_state", C.c_int, [_V, _I, _P, _P, _P, _P, _P]),
    ("uvlm_get_last_stats", C.c_int, [_V, C.POINTER(StepStats)]),
    ("uvlm_set_stage_timing", C.c_int, [_V, C.c_int32]),
    ("uvlm_synchronize", C.c_int, [_V]),
    ("uvlm_stream", _V, [_V]),
    ("uvlm_get_last_work", C.c_int, [_V, _P, _P, _P]),
    ("uvlm_velocity_at", C.c_int, [_V, _P, _I, C.c_int32, _P]),
    ("uvlm_kernel_launch_count", C.c_int64, []),
    ("uvlm_measure_fp32_peak", C.c_int, [C.c_int32, _P]),
    ("uvlm_measure_fp64_peak", C.c_int, [C.c_int32, _P]),
    ("uvlm_nbody_variant_name", C.c_char_p, [C.c_int32]),
    ("uvlm_sheet_induced_velocity", C.c_int, [_P, _P, _I, _I, _I, _P, _I, _P, C.c_int32]),
    ("uvlm_sheet_induced_velocity_noalloc", C.c_int, [_P, _P, _I, _I, _I, _P, _I, _P, C.c_int32, _V]),
    ("uvlm_advection_create", C.c_int, [C.c_char_p, C.c_int32, C.POINTER(_V)]),
    ("uvlm_advection_destroy", C.c_int, [_V]),
    ("uvlm_advection_advect", C.c_int, [_V, _P, _P, _P, _I, _I, _I, _P, _P, _I, _P, C.c_double]),
    ("uvlm_rings_induced_velocity", C.c_int, [_P, _P, _I, _P, _I, C.c_int32, _P]),
    ("uvlm_rings_advect", C.c_int, [_P, _P, _I, _P, _I, _P, C.c_double]),
    ("uvlm_rings_connect_trailing_edge", C.c_int, [_P, _I, _P]),
    ("uvlm_rings_solve_linear_problem", C.c_int, [_P, _P, _I, _P, _P, _I, _P, C.POINTER(Kinematics),
                                                  C.c_double, C.c_int32, _P]),
    ("uvlm_rings_solve_linear_problem_containers", C.c_int, [_P, _P, C.POINTER(C.c_int64), C.c_int32,
                                                             C.POINTER(Kinematics), _P, _P, _I, _P, C.c_double,
                                                             C.c_int32, _P]),
    ("uvlm_kinematics_perfome", C.c_int, [C.POINTER(Kinematics), _P, _I, C.c_double, _P]),
    ("uvlm_kinematics_velocity", C.c_int, [C.POINTER(Kinematics), _P, _I, C.c_double, _P]),
    ("uvlm_rings_load_katz_plotkin", C.c_int, [_P, _P, _P, _I, _I, C.POINTER(Kinematics), _P, _P, _I, _P, _P, _I,
                                               _P, C.c_double, C.c_double, C.c_double, _P]),
    ("uvlm_rings_load_joukowski", C.c_int, [_P, _P, _P, _P, _I, _I, C.POINTER(Kinematics), _P, _P, _I, _P,
                                            C.c_double, C.c_double, C.c_double, _P]),
    ("uvlm_set_output_paths", C.c_int, [_V, C.c_char_p, C.c_char_p]),
    ("uvlm_flush_output", C.c_int, [_V]),
    ("uvlm_write_state_record", C.c_int, [C.c_char_p, C.c_int32, C.c_int32, _I, _I, _I, _I, _P, _P, _P, _P,
                                          C.c_double]),
    ("uvlm_write_legacy_snapshot2", C.c_int, [C.c_char_p, C.c_double, _I, C.POINTER(C.c_int64),
                                              C.POINTER(C.c_int64), _P, _P, _P, _P, _P, _I, _P, _P, _P, _I]),
    ("uvlm_rings_vortex_impulse", C.c_int, [_P, _P, _I, _P]),
    ("uvlm_rings_lamb_vector", C.c_int, [_P, _P, _P, _I, _P, _P, _P, _I, _P]),
    ("uvlm_mlp_create", C.c_int, [C.c_uint64, C.POINTER(_V)]),
    ("uvlm_mlp_destroy", C.c_int, [_V]),
    ("uvlm_mlp_num_params", C.c_int64, [_V]),
    ("uvlm_mlp_get_params", C.c_int, [_V, C.POINTER(C.c_float)]),
    ("uvlm_mlp_set_params", C.c_int, [_V, C.POINTER(C.c_float)]),
    ("uvlm_mlp_set_normalization", C.c_int, [_V, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float]),
    ("uvlm_mlp_forward", C.c_int, [_V, C.POINTER(C.c_float), _I, C.POINTER(C.c_float)]),
    ("uvlm_mlp_forward_tc", C.c_int, [_V, C.POINTER(C.c_float), _I, C.POINTER(C.c_float)]),
    ("uvlm_mlp_gradients", C.c_int, [_V, C.POINTER(C.c_float), C.POINTER(C.c_float), _I, C.POINTER(C.c_float),
                                     _P]),
    ("uvlm_mlp_train", C.c_int, [_V, C.POINTER(C.c_float), C.POINTER(C.c_float), _I, C.c_int32, C.c_int32,
                                 C.c_double, C.c_uint64, _P]),
    ("uvlm_set_mlp", C.c_int, [_V, _V]),
    ("uvlm_collect_training_data", C.c_int, [_V, C.c_int32, _I]),
    ("uvlm_get_training_data", C.c_int, [_V, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(_I)]),
    ("uvlm_lu_factor_f32", C.c_int, [C.POINTER(C.c_float), _I, C.c_int32, C.POINTER(C.c_float),
                                     C.POINTER(C.c_int32)]),
    ("uvlm_dense_solve", C.c_int, [_P, _I, _P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    ("uvlm_batch_config_default", C.c_int, [C.POINTER(BatchConfig)]),
    ("uvlm_batch_create", C.c_int, [C.POINTER(BatchConfig), C.POINTER(BatchCase), C.c_int32, C.POINTER(_V)]),
    ("uvlm_batch_nbody_tile_name", C.c_char_p, [_V]),
    ("uvlm_batch_destroy", C.c_int, [_V]),
    ("uvlm_batch_last_error", C.c_char_p, [_V]),
    ("uvlm_batch_run", C.c_int, [_V, _I]),
    ("uvlm_batch_steps_done", C.c_int, [_V, C.POINTER(_I)]),
    ("uvlm_batch_get_loads", C.c_int, [_V, _P]),
    ("uvlm_batch_get_case", C.c_int, [_V, C.c_int32, _P, _P, _P, _P, C.POINTER(_I)]),
    ("uvlm_batch_get_solve_stats", C.c_int, [_V, C.POINTER(C.c_int32), _P]),
    ("uvlm_batch_launches_per_step", C.c_int, [_V, C.POINTER(_I)]),
    ("uvlm_batch_factorizations", C.c_int, [_V, C.POINTER(_I)]),
    ("uvlm_batch_stream", _V, [_V]),
]

_lib = None


def ensure_built() -> str:
    if not os.path.exists(LIB_PATH):
        from . import build as _b  # nvcc is part of the image; builds in-tree

        _b.build()
    return LIB_PATH


def lib():
    """The loaded C-ABI library (built in-tree on first use if absent)."""
    global _lib
    if _lib is None:
        path = ensure_built()
        L = C.CDLL(path)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class UVLMError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def check(code: int, ctx=None):
    if code != UVLM_OK:
        if ctx is not None:
            msg = lib().uvlm_last_error(ctx)
        else:
            msg = lib().uvlm_global_last_error()
        raise UVLMError(code, (msg or b"").decode())
