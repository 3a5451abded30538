"""Legacy AoS vortex-ring API (src/shed.h:14-46, src/linear.h:104-119).

Rings are arrays of shape (n, 4, 3): VortexRing::nodes() of each ring.  The
segments of a ring run nodes[k+1] -> nodes[k] (ForEachSegment,
src/vortex.h:132-140).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import check, lib

_P = C.POINTER(C.c_double)


def _p(a):
    return None if a is None or a.size == 0 else a.ctypes.data_as(_P)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def InducedVelocity(pos, rings, gammas, chordwise: bool = False) -> np.ndarray:  # noqa: N802
    """UVLM::InducedVelocity / ChordwiseInducedVelocity (src/shed.inl:22-33, 66-77)."""
    r = _f64(rings).reshape(-1, 4, 3)
    g = _f64(gammas).reshape(-1)
    x = _f64(pos)
    single = x.ndim == 1
    x = x.reshape(-1, 3)
    out = np.zeros_like(x)
    check(lib().uvlm_rings_induced_velocity(_p(r), _p(g), r.shape[0], _p(x), x.shape[0], int(chordwise), _p(out)))
    return out[0] if single else out


def AdvectParallel(vortex_rings, vortex_gammas, wake_rings, freestream, dt) -> np.ndarray:  # noqa: N802
    """UVLM::AdvectParallel (src/shed.inl:52-64); returns the moved wake rings."""
    v = _f64(vortex_rings).reshape(-1, 4, 3)
    g = _f64(vortex_gammas).reshape(-1)
    w = _f64(wake_rings).reshape(-1, 4, 3).copy()
    check(lib().uvlm_rings_advect(_p(v), _p(g), v.shape[0], _p(w), w.shape[0], _p(_f64(freestream)), float(dt)))
    return w


Advect = AdvectParallel


def ConnectTrailingEdge(edge_rings, wake_rings) -> np.ndarray:  # noqa: N802
    """UVLM::ConnectTrailingEdge (src/shed.inl:79-86)."""
    e = _f64(edge_rings).reshape(-1, 4, 3)
    w = _f64(wake_rings).reshape(-1, 4, 3).copy()
    check(lib().uvlm_rings_connect_trailing_edge(_p(e), e.shape[0], _p(w)))
    return w


def SolveLinearProblem(bound_rings, wake_rings, wake_gammas, freestream, morphing, t,  # noqa: N802
                       drop_wake_term: bool = True, bound_rings0=None) -> np.ndarray:
    """UVLM::SolveLinearProblem (src/linear.inl:113-130).

    drop_wake_term=True reproduces the reference, whose wake RHS term is a
    discarded statement (src/linear.inl:123-124)."""
    b = _f64(bound_rings).reshape(-1, 4, 3)
    b0 = None if bound_rings0 is None else _f64(bound_rings0).reshape(-1, 4, 3)
    w = _f64(wake_rings).reshape(-1, 4, 3)
    wg = _f64(wake_gammas).reshape(-1)
    out = np.zeros(b.shape[0])
    check(lib().uvlm_rings_solve_linear_problem(_p(b), _p(b0), b.shape[0], _p(w), _p(wg), w.shape[0],
                                                _p(_f64(freestream)), C.byref(morphing.k), float(t),
                                                int(drop_wake_term), _p(out)))
    return out


def CalcVortexImpulse(rings, gammas) -> np.ndarray:  # noqa: N802
    """Sum of VortexRing::Impulse() over the rings (calc_impulse_main.cpp:34-41, vortex.cpp:140-143)."""
    r = _f64(rings).reshape(-1, 4, 3)
    g = _f64(gammas).reshape(-1)
    out = np.zeros(3)
    check(lib().uvlm_rings_vortex_impulse(_p(r), _p(g), r.shape[0], out.ctypes.data_as(_P)))
    return out


def CalcLambVector(panels, panel_gammas, node_velocities, freestream, vortices, vortex_gammas) -> np.ndarray:  # noqa: N802
    """Sum over panels of calc_impulse::CalcLambVectorOnPanel (calc_impulse.h:15-30), as
    calc_impulse_main.cpp:79-82 sums it.  node_velocities: (n, 4, 3), one per segment in
    ForEachSegment order; freestream: one 3-vector or one per panel."""
    p = _f64(panels).reshape(-1, 4, 3)
    g = _f64(panel_gammas).reshape(-1)
    v = _f64(node_velocities).reshape(-1, 4, 3)
    fs = np.ascontiguousarray(np.broadcast_to(_f64(freestream).reshape(-1, 3), (p.shape[0], 3)))
    w = _f64(vortices).reshape(-1, 4, 3)
    wg = _f64(vortex_gammas).reshape(-1)
    out = np.zeros(3)
    check(lib().uvlm_rings_lamb_vector(_p(p), _p(g), _p(v), p.shape[0], _p(fs), _p(w), _p(wg), w.shape[0],
                                       out.ctypes.data_as(_P)))
    return out


def _kin(morphing):
    return morphing.k if hasattr(morphing, "k") else morphing


def SolveLinearProblemContainers(bound_rings, container_rings, morphings, wake_rings, wake_gammas, freestream, t,  # noqa: N802
                                 drop_wake_term: bool = True, bound_rings0=None) -> np.ndarray:
    """UVLM::SolveLinearProblem(containers, morphings, freestream, t) (src/linear.inl:132-157): the bound rings
    of the containers one after another (container c: container_rings[c] rings, moving with morphings[c]),
    then the wake rings."""
    from ._capi import Kinematics

    b = _f64(bound_rings).reshape(-1, 4, 3)
    b0 = None if bound_rings0 is None else _f64(bound_rings0).reshape(-1, 4, 3)
    w = _f64(wake_rings).reshape(-1, 4, 3)
    wg = _f64(wake_gammas).reshape(-1)
    sizes = (C.c_int64 * len(container_rings))(*[int(c) for c in container_rings])
    kins = (Kinematics * len(morphings))(*[_kin(m) for m in morphings])
    out = np.zeros(b.shape[0])
    check(lib().uvlm_rings_solve_linear_problem_containers(_p(b), _p(b0), sizes, len(morphings), kins, _p(w), _p(wg),
                                                           w.shape[0], _p(_f64(freestream)), float(t),
                                                           int(drop_wake_term), _p(out)))
    return out


def CalcLoadKatzPlotkin(rings, gammas, gammas_prev, rows, cols, morphing, freestream, rho, t, dt,  # noqa: N802
                        bound_rings=None, bound_gammas=None, wake_rings=None, wake_gammas=None) -> np.ndarray:
    """calc_load::CalcLoadKatzPlotkin (src/calc_load/katz_plotkin.cpp:16-68) for one container of rows x cols
    rings; returns F.x, F.y, F.z, Pin, Pout.  The UVLMVortexRing argument is given by its bound rings
    (chordwise velocity) and wake rings; leave them None for the empty one of the legacy simulator."""
    r = _f64(rings).reshape(-1, 4, 3)
    b = np.zeros((0, 4, 3)) if bound_rings is None else _f64(bound_rings).reshape(-1, 4, 3)
    bg = np.zeros(0) if bound_gammas is None else _f64(bound_gammas).reshape(-1)
    w = np.zeros((0, 4, 3)) if wake_rings is None else _f64(wake_rings).reshape(-1, 4, 3)
    wg = np.zeros(0) if wake_gammas is None else _f64(wake_gammas).reshape(-1)
    out = np.zeros(5)
    check(lib().uvlm_rings_load_katz_plotkin(_p(r), _p(_f64(gammas)), _p(_f64(gammas_prev)), int(rows), int(cols),
                                             C.byref(_kin(morphing)), _p(b), _p(bg), b.shape[0], _p(w), _p(wg),
                                             w.shape[0], _p(_f64(freestream)), float(rho), float(t), float(dt),
                                             out.ctypes.data_as(_P)))
    return out


def CalcLoadJoukowski(rings, rings0, gammas, gammas_prev, rows, cols, morphing, vortices, vortex_gammas,  # noqa: N802
                      freestream, rho, t, dt) -> np.ndarray:
    """Container calc_load::CalcLoadJoukowski (src/calc_load/joukowski.h:24-104): rings / rings0 are the
    container's nodes() / nodes0(), `vortices` its whole ring pool; returns F.x, F.y, F.z, Pin, Pout."""
    r = _f64(rings).reshape(-1, 4, 3)
    v = _f64(vortices).reshape(-1, 4, 3)
    out = np.zeros(5)
    check(lib().uvlm_rings_load_joukowski(_p(r), _p(_f64(rings0)), _p(_f64(gammas)), _p(_f64(gammas_prev)),
                                          int(rows), int(cols), C.byref(_kin(morphing)), _p(v),
                                          _p(_f64(vortex_gammas)), v.shape[0], _p(_f64(freestream)), float(rho),
                                          float(t), float(dt), out.ctypes.data_as(_P)))
    return out
