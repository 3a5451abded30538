"""The legacy stepper (src/simulator/simulator.cpp:220-270) restated over the FP64 CPU oracle.

TEST INFRASTRUCTURE ONLY: only ``tests/`` may import this module.  It
composes the oracle's restatements of the reference's ring primitives
(``uvlm_oracle.cpp``: Morphing::Perfome, SolveLinearProblem over containers,
CalcLoadKatzPlotkin, the container CalcLoadJoukowski, AdvectParallel) in
the order of the reference's main loop, on the same pool layout (bound rings
of every wing, then wake rings, newest wake row first).
"""
from __future__ import annotations

import numpy as np

import pyoracle as o


def container_rings(points, rows, cols, origin):
    """WingBuilder::AddWing + BuildWing (src/wing_builder.cpp:12-76) with TransformRow
    (src/wing_builder.h:21-35): mirror each half-wing point row, then ring (i, j) =
    p(i, j), p(i+1, j), p(i+1, j+1), p(i, j+1)."""
    pts = np.asarray(points, float).reshape(rows + 1, cols + 1, 3)
    full = []
    for i in range(rows + 1):
        row = pts[i]
        mir = np.array([[p[0], -p[1], p[2]] for p in row[1:][::-1]])
        full.append(np.concatenate([mir, row]) + np.asarray(origin, float))
    P = np.array(full)
    out = []
    for i in range(rows):
        for j in range(2 * cols):
            out.append([P[i, j], P[i + 1, j], P[i + 1, j + 1], P[i, j + 1]])
    return np.array(out)


def start(wings, kins, inlet, steps, dt, use_joukowski=False, disable_wake=False, drop_wake_term=True):
    """simulator::Start.  wings: list of dicts (rows, cols, points, origin, chord, span) of half-wing
    descriptions; kins: oracle Kinematics per wing, their origin set to the wing's (simulator.cpp:205-209)."""
    blocks = [container_rings(w["points"], w["rows"], w["cols"], w["origin"]) for w in wings]
    shapes = [(w["rows"], 2 * w["cols"]) for w in wings]
    sizes = [r * c for r, c in shapes]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(int)
    bound0 = np.concatenate(blocks)
    bound = bound0.copy()
    g = np.zeros(len(bound))
    wake = np.zeros((0, 4, 3))
    wg = np.zeros(0)
    inlet = np.asarray(inlet, float)
    r0, c0 = shapes[0]
    edge = slice((r0 - 1) * c0, r0 * c0)
    rows_out = []
    for step in range(steps + 1):
        t = dt * step
        g_prev = g.copy()
        # MorphingProcess (simulator.cpp:99-108): nodes = Perfome(nodes0)
        for c, k in enumerate(kins):
            for q in range(offs[c], offs[c + 1]):
                for n in range(4):
                    bound[q, n] = o.perfome(k, bound0[q, n], t)
        # ConnectProcess (:82-97)
        if len(wake) >= c0:
            wake[:c0, 0] = bound[edge, 1]
            wake[:c0, 3] = bound[edge, 2]
        g = o.solve_linear_problem_containers(bound, sizes, kins, wake, wg, inlet, t, drop_wake_term, bound0)
        row = [t]
        pool = np.concatenate([bound, wake])
        pool_g = np.concatenate([g, wg])
        U = np.linalg.norm(inlet)
        for c, (w, k) in enumerate(zip(wings, kins)):
            a, b = offs[c], offs[c + 1]
            rows, cols = shapes[c]
            if use_joukowski:
                load = o.load_joukowski_rings(bound[a:b], bound0[a:b], g[a:b], g_prev[a:b], rows, cols, k, pool,
                                              pool_g, inlet, 1.0, t, dt)
            else:
                load = o.load_katz_plotkin(bound[a:b], g[a:b], g_prev[a:b], rows, cols, k, inlet, 1.0, t, dt)
            coeff = load[:3] / (0.5 * U * U * w["chord"] * w["span"])
            row += list(coeff) + [load[3], load[4]]
        rows_out.append(row)
        if step == steps:
            break
        if not disable_wake:
            # shed the first wing's trailing edge and roll the wake up (:252-266)
            wake_next = np.concatenate([bound[edge], wake])
            wg_next = np.concatenate([g[edge], wg])
            wake = o.rings_advect(pool, pool_g, wake_next, inlet, dt, parallel=True)
            wg = wg_next
    return np.array(rows_out)
