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


def morphing_velocities(bound0, offs, kins, inlet, t):
    """OutputSnapshot2's MorphingVelocity records (simulator.cpp:135-152): per bound ring, Morphing::Velocity
    at the reference centroid (src/vortex.cpp:102-104) and at (start0 + end0) / 2 of each segment,
    start0 = nodes0[(q + 1) % 4], end0 = nodes0[q] (src/vortex.h:149-160), and the inlet."""
    center, nodes = [], []
    for c, k in enumerate(kins):
        for r in bound0[offs[c]:offs[c + 1]]:
            center.append(o.morph_velocity(k, (r[0] + r[1] + r[2] + r[3]) / 4, t))
            nodes.append([o.morph_velocity(k, (r[(q + 1) % 4] + r[q]) / 2, t) for q in range(4)])
    n = len(center)
    return np.array(center).reshape(n, 3), np.array(nodes).reshape(n, 4, 3), np.tile(inlet, (n, 1))


def start(wings, kins, inlet, steps, dt, use_joukowski=False, disable_wake=False, drop_wake_term=True,
          snapshots=None):
    """simulator::Start.  wings: list of dicts (rows, cols, points, origin, chord, span) of half-wing
    descriptions; kins: oracle Kinematics per wing, their origin set to the wing's (simulator.cpp:205-209).
    A list given as `snapshots` receives, per step, the content of OutputSnapshot2 (:118-160): t, the ring
    pool with its reference nodes and circulations, and the morphing velocity records."""
    blocks = [container_rings(w["points"], w["rows"], w["cols"], w["origin"]) for w in wings]
    shapes = [(w["rows"], 2 * w["cols"]) for w in wings]
    sizes = [r * c for r, c in shapes]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(int)
    bound0 = np.concatenate(blocks)
    bound = bound0.copy()
    g = np.zeros(len(bound))
    wake = np.zeros((0, 4, 3))
    wake0 = np.zeros((0, 4, 3))
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
        if snapshots is not None:
            mc, mn, mf = morphing_velocities(bound0, offs, kins, inlet, t)
            snapshots.append(dict(t=t, rings=np.concatenate([bound, wake]), rings0=np.concatenate([bound0, wake0]),
                                  gammas=np.concatenate([g, wg]), mv_center=mc, mv_nodes=mn, mv_freestream=mf))
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
            wake0 = np.concatenate([bound0[edge], wake0])  # shed rings carry the edge rings' nodes0
            wg = wg_next
    return np.array(rows_out)


def calc_impulse(snap):
    """CalcImpulse (src/calc_impulse_main.cpp:54-87) over a decoded legacy Snapshot2, ring by ring on the
    oracle: [t, impulse of container 0, its Lamb-vector term, impulse of the wake]."""
    shapes = snap["container_shapes"]
    c0 = shapes[0]
    n0 = c0["rows"] * c0["cols"]
    a = c0["id"] * n0
    n_bound = sum(c["rows"] * c["cols"] for c in shapes)
    R, G = snap["rings"], snap["gammas"]
    imp = o.vortex_impulse(R[a:a + n0], G[a:a + n0])
    wake = o.vortex_impulse(R[n_bound:], G[n_bound:]) if len(R) > n_bound else np.zeros(3)
    other = o.lamb_vector(R[a:a + n0], G[a:a + n0], snap["mv_nodes"][:n0], snap["mv_freestream"][:n0], R, G)
    return np.concatenate([[snap["t"]], imp, other, wake])
