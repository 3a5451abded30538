"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the FP64 CPU restatement of xeno14/UVLM's time-stepper in
``oracle/uvlm_oracle.cpp``.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference arm may import this module; the
product (``uvlm_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class Kinematics(C.Structure):
    """Closed-form Morphing parameters (layout of orc_kinematics)."""

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


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_P = C.POINTER(C.c_double)
_I = C.c_int64


def _declare(L):
    L.orc_biot_savart.argtypes = [_P, _P, _P, _P]
    L.orc_distance_line_and_point.argtypes = [_P, _P, _P]
    L.orc_distance_line_and_point.restype = C.c_double
    L.orc_voring.argtypes = [_P, _I, _I, _I, _P, _I, _I, _I, _I, _I, _P, _P]
    L.orc_sheet_induced_velocity.argtypes = [_P, _I, _I, _I, _P, _I, _I, _P, _I, _P]
    L.orc_ring_biot_savart.argtypes = [_P, C.c_double, _P, _P]
    L.orc_ring_chordwise_biot_savart.argtypes = [_P, C.c_double, _P, _P]
    L.orc_ring_vector.argtypes = [_P, C.c_double, C.c_int, _P]
    L.orc_ring_scalar.argtypes = [_P, C.c_int]
    L.orc_ring_scalar.restype = C.c_double
    L.orc_solve_linear_problem_containers.argtypes = [_P, _P, C.POINTER(C.c_int64), C.c_int,
                                                      C.POINTER(Kinematics), _P, _P, _I, _P, C.c_double, C.c_int,
                                                      _P]
    L.orc_solve_linear_problem_containers.restype = C.c_int
    L.orc_load_katz_plotkin.argtypes = [_P, _P, _P, _I, _I, C.POINTER(Kinematics), _P, _P, _I, _P, _P, _I, _P,
                                        C.c_double, C.c_double, C.c_double, _P]
    L.orc_load_katz_plotkin.restype = None
    L.orc_load_joukowski_rings.argtypes = [_P, _P, _P, _P, _I, _I, C.POINTER(Kinematics), _P, _P, _I, _P,
                                           C.c_double, C.c_double, C.c_double, _P]
    L.orc_load_joukowski_rings.restype = None
    L.orc_vortex_impulse.argtypes = [_P, _P, _I, _P]
    L.orc_vortex_impulse.restype = None
    L.orc_lamb_vector.argtypes = [_P, _P, _P, _I, _P, _P, _P, _I, _P]
    L.orc_lamb_vector.restype = None
    L.orc_ring_angle_of_attack.argtypes = [_P, _P]
    L.orc_ring_angle_of_attack.restype = C.c_double
    L.orc_rings_induced_velocity.argtypes = [_P, _P, _I, _P, C.c_int, _P]
    L.orc_rings_advect.argtypes = [_P, _P, _I, _P, _I, _P, C.c_double, C.c_int]
    L.orc_connect_trailing_edge.argtypes = [_P, _I, _P]
    L.orc_solve_linear_problem.argtypes = [_P, _P, _I, _P, _P, _I, _P, C.POINTER(Kinematics),
                                           C.c_double, C.c_int, _P]
    L.orc_calc_morphing_velocity_on_wing.argtypes = [_P, _P, _I, C.POINTER(Kinematics), C.c_double, _P]
    L.orc_kin_perfome.argtypes = [C.POINTER(Kinematics), _P, C.c_double, _P]
    L.orc_kin_velocity.argtypes = [C.POINTER(Kinematics), _P, C.c_double, C.c_double, _P]
    L.orc_calc_um.argtypes = [C.POINTER(Kinematics), _P, _P, C.c_double, _P]
    L.orc_transform_chebyshev.argtypes = [_I, C.c_double, C.c_double, _P]
    L.orc_rect_generate.argtypes = [C.c_double, C.c_double, _I, _I, C.c_int, C.c_int, _P]
    L.orc_whole_wing.argtypes = [_P, _I, _I, _P, _P]
    L.orc_fullpiv_lu_solve.argtypes = [_P, _I, _P, _P]
    L.orc_sim_create.restype = C.c_void_p
    L.orc_sim_destroy.argtypes = [C.c_void_p]
    L.orc_sim_add_wing.argtypes = [C.c_void_p, C.c_double, C.c_double, _I, _I, _P,
                                   C.POINTER(Kinematics), C.c_int, C.c_int]
    L.orc_sim_set_forward_flight.argtypes = [C.c_void_p, _P]
    L.orc_sim_set_advection.argtypes = [C.c_void_p, C.c_char_p]
    L.orc_sim_set_erase_wake_after.argtypes = [C.c_void_p, _I]
    L.orc_sim_set_threads.argtypes = [C.c_void_p, C.c_int]
    L.orc_sim_begin.argtypes = [C.c_void_p]
    L.orc_sim_step.argtypes = [C.c_void_p, _I, C.c_double, _P]
    L.orc_sim_sizes.argtypes = [C.c_void_p, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]
    L.orc_sim_wake_node_rows.argtypes = [C.c_void_p]
    L.orc_sim_wake_node_rows.restype = _I
    L.orc_sim_get_state.argtypes = [C.c_void_p, _P, _P, _P, _P, _P, _P]
    L.orc_sim_set_state.argtypes = [C.c_void_p, _I, _P, _P, _P, _P, _P]
    L.orc_sim_time_step_sampled.argtypes = [C.c_void_p, _I, C.c_double, _I, _I, _P]
    L.orc_sim_add_wing_generator.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, _I, _I, _P,
                                             C.POINTER(Kinematics), C.c_int, C.c_int]
    L.orc_naca4digit.argtypes = [C.c_double, C.c_double, C.c_int]
    L.orc_naca4digit.restype = C.c_double
    L.orc_naca00xx.argtypes = [C.c_double, C.c_double, C.c_int]
    L.orc_naca00xx.restype = C.c_double
    L.orc_generate_wing.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _I, _I, C.c_int, C.c_int, _P]
    L.orc_sim_set_lu_threads.argtypes = [C.c_void_p, C.c_int]
    L.orc_sim_sliced_begin.argtypes = [C.c_void_p, _I, C.c_double, _I, C.c_int]
    L.orc_sim_sliced_run.argtypes = [C.c_void_p, _I, _P]


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_P)


def _v(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def kinematics(**kw) -> Kinematics:
    k = Kinematics()
    for name, val in kw.items():
        if name == "origin":
            for i in range(3):
                k.origin[i] = float(val[i])
        else:
            setattr(k, name, float(val))
    return k


# ---------------------------------------------------------------- primitives
def biot_savart(start, end, pos):
    out = np.zeros(3)
    lib().orc_biot_savart(_p(_v(start)), _p(_v(end)), _p(_v(pos)), _p(out))
    return out


def distance_line_and_point(start, end, pos):
    return lib().orc_distance_line_and_point(_p(_v(start)), _p(_v(end)), _p(_v(pos)))


def sheet_induced_velocity(pos, gamma, targets):
    """UVLM::InducedVelocity(x, pos, gamma) for each target (velocity.h:14-24).

    pos: (num, prows, pcols, 3); gamma: (num, grows, gcols); targets: (T, 3)."""
    pos = _v(pos)
    gamma = _v(gamma)
    targets = _v(targets).reshape(-1, 3)
    out = np.zeros_like(targets)
    pn, pr, pc = pos.shape[:3]
    _, gr, gc = gamma.shape
    lib().orc_sheet_induced_velocity(_p(pos), pn, pr, pc, _p(gamma), gr, gc, _p(targets),
                                     targets.shape[0], _p(out))
    return out


def ring_biot_savart(nodes, gamma, pos, chordwise=False):
    out = np.zeros(3)
    f = lib().orc_ring_chordwise_biot_savart if chordwise else lib().orc_ring_biot_savart
    f(_p(_v(nodes)), float(gamma), _p(_v(pos)), _p(out))
    return out


_VEC = {"normal": 0, "tangent": 1, "tangent2": 2, "centroid": 3, "tanvec_chord": 4,
        "tanvec_span": 5, "impulse": 6}
_SCA = {"area": 0, "c": 1, "b": 2}


def ring_vector(nodes, what, gamma=0.0):
    out = np.zeros(3)
    lib().orc_ring_vector(_p(_v(nodes)), float(gamma), _VEC[what], _p(out))
    return out


def ring_scalar(nodes, what):
    return lib().orc_ring_scalar(_p(_v(nodes)), _SCA[what])


def ring_angle_of_attack(nodes, Q):
    return lib().orc_ring_angle_of_attack(_p(_v(nodes)), _p(_v(Q)))


def rings_induced_velocity(rings, gammas, pos, chordwise=False):
    rings = _v(rings).reshape(-1, 4, 3)
    out = np.zeros(3)
    lib().orc_rings_induced_velocity(_p(rings), _p(_v(gammas)), rings.shape[0], _p(_v(pos)),
                                     int(chordwise), _p(out))
    return out


def rings_advect(vortex_rings, vortex_gamma, wake_rings, freestream, dt, parallel=True):
    vr = _v(vortex_rings).reshape(-1, 4, 3)
    wr = _v(wake_rings).reshape(-1, 4, 3).copy()
    vg = _v(vortex_gamma).reshape(-1)
    lib().orc_rings_advect(_p(vr) if vr.size else None, _p(vg) if vg.size else None, vr.shape[0],
                           _p(wr), wr.shape[0], _p(_v(freestream)), float(dt), int(parallel))
    return wr


def connect_trailing_edge(edge_rings, wake_rings):
    e = _v(edge_rings).reshape(-1, 4, 3)
    w = _v(wake_rings).reshape(-1, 4, 3).copy()
    lib().orc_connect_trailing_edge(_p(e), e.shape[0], _p(w))
    return w


def solve_linear_problem(bound_rings, wake_rings, wake_gamma, freestream, kin, t,
                         drop_wake_term=True, bound_rings0=None):
    b = _v(bound_rings).reshape(-1, 4, 3)
    b0 = b if bound_rings0 is None else _v(bound_rings0).reshape(-1, 4, 3)
    w = _v(wake_rings).reshape(-1, 4, 3)
    wg = _v(wake_gamma).reshape(-1)
    out = np.zeros(b.shape[0])
    rc = lib().orc_solve_linear_problem(_p(b), _p(b0), b.shape[0], _p(w) if w.size else None,
                                        _p(wg) if wg.size else None, w.shape[0], _p(_v(freestream)),
                                        C.byref(kin), float(t), int(drop_wake_term), _p(out))
    if rc:
        raise RuntimeError("singular matrix")
    return out


def calc_morphing_velocity_on_wing(rings, kin, t, rings0=None):
    r = _v(rings).reshape(-1, 4, 3)
    r0 = r if rings0 is None else _v(rings0).reshape(-1, 4, 3)
    out = np.zeros(r.shape[0])
    lib().orc_calc_morphing_velocity_on_wing(_p(r), _p(r0), r.shape[0], C.byref(kin), float(t), _p(out))
    return out


def perfome(kin, x0, t):
    out = np.zeros(3)
    lib().orc_kin_perfome(C.byref(kin), _p(_v(x0)), float(t), _p(out))
    return out


def morph_velocity(kin, x0, t, h=1e-6):
    out = np.zeros(3)
    lib().orc_kin_velocity(C.byref(kin), _p(_v(x0)), float(t), float(h), _p(out))
    return out


def calc_um(kin, x0, freestream, t):
    out = np.zeros(3)
    lib().orc_calc_um(C.byref(kin), _p(_v(x0)), _p(_v(freestream)), float(t), _p(out))
    return out


def transform_chebyshev(N, xmin, xmax):
    out = np.zeros(N)
    lib().orc_transform_chebyshev(N, float(xmin), float(xmax), _p(out))
    return out


def rect_generate(chord, span, rows, cols, cheb_chord=False, cheb_span=False):
    out = np.zeros(((rows + 1) * (cols + 1), 3))
    lib().orc_rect_generate(float(chord), float(span), rows, cols, int(cheb_chord), int(cheb_span), _p(out))
    return out


def whole_wing(half, rows, half_cols, origin=(0.0, 0.0, 0.0)):
    out = np.zeros(((rows + 1) * (2 * half_cols + 1), 3))
    lib().orc_whole_wing(_p(_v(half)), rows, half_cols, _p(_v(origin)), _p(out))
    return out


def fullpiv_lu_solve(A, b):
    A = _v(A).copy()
    b = _v(b)
    x = np.zeros(b.shape[0])
    rc = lib().orc_fullpiv_lu_solve(_p(A), A.shape[0], _p(b), _p(x))
    if rc:
        raise RuntimeError("singular matrix")
    return x


# ---------------------------------------------------------------- simulator
class Simulator:
    """SimpleSimulator restated on the CPU (simple_simulator.{h,cpp})."""

    def __init__(self):
        self._h = lib().orc_sim_create()
        self.num = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.orc_sim_destroy(h)
            self._h = None

    def add_wing(self, chord, span, rows, cols, origin=(0, 0, 0), kin=None,
                 cheb_chord=False, cheb_span=False):
        kin = kin if kin is not None else Kinematics()
        rc = lib().orc_sim_add_wing(self._h, float(chord), float(span), int(rows), int(cols),
                                    _p(_v(origin)), C.byref(kin), int(cheb_chord), int(cheb_span))
        if rc:
            raise ValueError(f"AddWing rejected the wing (code {rc})")
        self.num += 1

    def add_wing_generator(self, generator, digit, chord, span, rows, cols, origin=(0, 0, 0), kin=None,
                           cheb_chord=False, cheb_span=False):
        """AddWing with a NACA4digitGenerator(digit) ("naca4digit"), NACA00XXGenerator(digit) ("naca00xx") or
        RectGenerator ("rect") (simple_simulator.cpp:126-169)."""
        kin = kin if kin is not None else Kinematics()
        g = {"rect": 0, "naca4digit": 1, "naca00xx": 2}[generator]
        rc = lib().orc_sim_add_wing_generator(self._h, g, int(digit), float(chord), float(span), int(rows),
                                              int(cols), _p(_v(origin)), C.byref(kin), int(cheb_chord),
                                              int(cheb_span))
        if rc:
            raise ValueError(f"AddWing rejected the wing (code {rc})")
        self.num += 1

    def set_lu_threads(self, n):
        """Threads of the FullPivLU elimination (bit-identical for any count; 1 = Eigen's)."""
        lib().orc_sim_set_lu_threads(self._h, int(n))

    def sliced_begin(self, step, dt, slices, threads):
        """Plans MainLoop(step, dt) as `slices` consecutive slices of about equal estimated time."""
        rc = lib().orc_sim_sliced_begin(self._h, int(step), float(dt), int(slices), int(threads))
        if rc:
            raise RuntimeError(f"sliced_begin failed ({rc})")

    def sliced_run(self, slice_index, row=None):
        """Runs one slice; all slices in order perform exactly step(step, dt).  `row` (1 + 2 num doubles)
        receives the load row when the slice finishes the loads."""
        rc = lib().orc_sim_sliced_run(self._h, int(slice_index), _p(row))
        if rc:
            raise RuntimeError(f"sliced_run failed ({rc})")

    def set_forward_flight(self, ff):
        lib().orc_sim_set_forward_flight(self._h, _p(_v(ff)))

    def set_advection(self, name):
        if lib().orc_sim_set_advection(self._h, name.encode()):
            raise ValueError(name)

    def set_erase_wake_after(self, step):
        lib().orc_sim_set_erase_wake_after(self._h, int(step))

    def set_threads(self, n):
        lib().orc_sim_set_threads(self._h, int(n))

    def begin(self):
        rc = lib().orc_sim_begin(self._h)
        if rc:
            raise RuntimeError(f"begin failed ({rc})")

    def step(self, step, dt):
        row = np.zeros(1 + 2 * self.num)
        rc = lib().orc_sim_step(self._h, int(step), float(dt), _p(row))
        if rc:
            raise RuntimeError(f"step failed ({rc})")
        return row

    def run(self, steps, dt):
        self.begin()
        return np.stack([self.step(s, dt) for s in range(steps + 1)])

    def sizes(self):
        a, b, c, d = _I(), _I(), _I(), _I()
        lib().orc_sim_sizes(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return a.value, b.value, c.value, d.value

    def state(self):
        num, rows, cols, wr = self.sizes()
        s = dict(
            wing_pos=np.zeros((num, rows + 1, cols + 1, 3)),
            wing_pos_init=np.zeros((num, rows + 1, cols + 1, 3)),
            wake_pos=np.zeros((num, lib().orc_sim_wake_node_rows(self._h), cols + 1, 3)),
            wing_gamma=np.zeros((num, rows, cols)),
            wing_gamma_prev=np.zeros((num, rows, cols)),
            wake_gamma=np.zeros((num, wr, cols)),
        )
        lib().orc_sim_get_state(self._h, _p(s["wing_pos"]), _p(s["wing_pos_init"]),
                                _p(s["wake_pos"]), _p(s["wing_gamma"]), _p(s["wing_gamma_prev"]),
                                _p(s["wake_gamma"]))
        return s

    def set_state(self, wake_rows, wing_pos, wake_pos, wing_gamma, wing_gamma_prev, wake_gamma):
        rc = lib().orc_sim_set_state(self._h, int(wake_rows), _p(_v(wing_pos)), _p(_v(wake_pos)),
                                     _p(_v(wing_gamma)), _p(_v(wing_gamma_prev)), _p(_v(wake_gamma)))
        if rc:
            raise RuntimeError("set_state failed")

    def time_step_sampled(self, step, dt, stride, lu_n):
        sec = np.zeros(6)
        rc = lib().orc_sim_time_step_sampled(self._h, int(step), float(dt), int(stride), int(lu_n), _p(sec))
        if rc:
            raise RuntimeError("time_step_sampled failed")
        return sec


def naca4digit(x, c, xx):
    """Mean camber of a 4-digit NACA section (src/wing/naca4digit.cpp:12-27)."""
    return lib().orc_naca4digit(float(x), float(c), int(xx))


def naca00xx(x, c, xx):
    """Half thickness of a symmetric 4-digit NACA section (src/wing/naca00XX.cpp:14-19)."""
    return lib().orc_naca00xx(float(x), float(c), int(xx))


def generate_wing(generator, digit, chord, span, rows, cols, cheb_chord=False, cheb_span=False):
    """WingGenerator::Generate points of "rect", "naca4digit" or "naca00xx": (rows+1, cols+1, 3)."""
    g = {"rect": 0, "naca4digit": 1, "naca00xx": 2}[generator]
    out = np.zeros((rows + 1, cols + 1, 3))
    lib().orc_generate_wing(g, int(digit), float(chord), float(span), int(rows), int(cols), int(cheb_chord),
                            int(cheb_span), _p(out))
    return out


def vortex_impulse(rings, gammas):
    """Sum of VortexRing::Impulse() over AoS rings (calc_impulse_main.cpp:34-41)."""
    rings = _v(rings).reshape(-1, 12)
    out = np.zeros(3)
    lib().orc_vortex_impulse(_p(rings), _p(_v(gammas)), rings.shape[0], _p(out))
    return out


def lamb_vector(panels, panel_gamma, v_nodes, freestream, vortices, vortex_gamma):
    """Sum over panels of CalcLambVectorOnPanel (calc_impulse.h:15-30); freestream is one 3-vector or one per
    panel (calc_impulse_main.cpp:79-82)."""
    panels = _v(panels).reshape(-1, 12)
    fs = np.ascontiguousarray(np.broadcast_to(_v(freestream).reshape(-1, 3), (panels.shape[0], 3)))
    vortices = _v(vortices).reshape(-1, 12)
    out = np.zeros(3)
    lib().orc_lamb_vector(_p(panels), _p(_v(panel_gamma)), _p(_v(v_nodes).reshape(-1, 12)), panels.shape[0],
                          _p(fs), _p(vortices) if vortices.size else None,
                          _p(_v(vortex_gamma)) if vortices.size else None, vortices.shape[0], _p(out))
    return out


def _opt(a):
    return _p(a) if a is not None and a.size else None


def solve_linear_problem_containers(bound_rings, container_rings, kins, wake_rings, wake_gamma, freestream, t,
                                    drop_wake_term=True, bound_rings0=None):
    """SolveLinearProblem(containers, morphings, freestream, t) (src/linear.inl:132-157)."""
    b = _v(bound_rings).reshape(-1, 4, 3)
    b0 = b if bound_rings0 is None else _v(bound_rings0).reshape(-1, 4, 3)
    w = _v(wake_rings).reshape(-1, 4, 3)
    wg = _v(wake_gamma).reshape(-1)
    sizes = (C.c_int64 * len(container_rings))(*[int(c) for c in container_rings])
    karr = (Kinematics * len(kins))(*kins)
    out = np.zeros(b.shape[0])
    rc = lib().orc_solve_linear_problem_containers(_p(b), _p(b0), sizes, len(kins), karr, _opt(w), _opt(wg),
                                                   w.shape[0], _p(_v(freestream)), float(t), int(drop_wake_term),
                                                   _p(out))
    if rc:
        raise RuntimeError("singular matrix")
    return out


def load_katz_plotkin(rings, gamma, gamma_prev, rows, cols, kin, freestream, rho, t, dt, bound_rings=None,
                      bound_gamma=None, wake_rings=None, wake_gamma=None):
    """CalcLoadKatzPlotkin (src/calc_load/katz_plotkin.cpp:16-68) -> (F, Pin, Pout) as 5 numbers."""
    r = _v(rings).reshape(-1, 4, 3)
    b = np.zeros((0, 4, 3)) if bound_rings is None else _v(bound_rings).reshape(-1, 4, 3)
    bg = np.zeros(0) if bound_gamma is None else _v(bound_gamma).reshape(-1)
    w = np.zeros((0, 4, 3)) if wake_rings is None else _v(wake_rings).reshape(-1, 4, 3)
    wg = np.zeros(0) if wake_gamma is None else _v(wake_gamma).reshape(-1)
    out = np.zeros(5)
    lib().orc_load_katz_plotkin(_p(r), _p(_v(gamma)), _p(_v(gamma_prev)), int(rows), int(cols), C.byref(kin),
                                _opt(b), _opt(bg), b.shape[0], _opt(w), _opt(wg), w.shape[0], _p(_v(freestream)),
                                float(rho), float(t), float(dt), _p(out))
    return out


def load_joukowski_rings(rings, rings0, gamma, gamma_prev, rows, cols, kin, vortices, vortex_gamma, freestream,
                         rho, t, dt):
    """Container CalcLoadJoukowski (src/calc_load/joukowski.h:24-104) -> (F, Pin, Pout) as 5 numbers."""
    r = _v(rings).reshape(-1, 4, 3)
    v = _v(vortices).reshape(-1, 4, 3)
    out = np.zeros(5)
    lib().orc_load_joukowski_rings(_p(r), _p(_v(rings0)), _p(_v(gamma)), _p(_v(gamma_prev)), int(rows), int(cols),
                                   C.byref(kin), _opt(v), _opt(_v(vortex_gamma)), v.shape[0], _p(_v(freestream)),
                                   float(rho), float(t), float(dt), _p(out))
    return out
