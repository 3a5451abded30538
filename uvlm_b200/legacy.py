"""The reference's legacy stepper (src/simulator/simulator.{h,cpp}) over AoS vortex rings.

The legacy API keeps every ring of every wing and of the wake in one pool of
`VortexRing`s (src/vortex_container.h:22-136); a `VortexContainer` is a
rows x cols view of a wing's bound rings in it.  `LegacySimulator.Start`
runs the legacy main loop (simulator.cpp:220-270): Morphing of the bound
rings and reconnection of the newest wake row to the trailing edge
(:82-108), the circulation solve of linear.inl (:110-116), the loads of the
chosen formulation (:162-200), then shedding and roll-up of the wake by
AdvectParallel (:252-266).  Each stage is one call of the C-ABI (the CUDA
kernels); the host only moves the AoS arrays.  With `SetOutputPath(dir)`
every step writes `dir/%08d`, one unframed Snapshot2 (OutputSnapshot2,
:118-160): the container shapes, the whole ring pool with its reference
nodes and, per bound ring, the morphing velocity at its reference centroid
and at the reference midpoint of each segment, with the inlet.  With
`SetOutputLoadPath(path)` the load rows are appended to path, tab-joined
(CalcLoadProcess :162-200).  Containers are packed one after another; this
is the reference's layout (container c at c x rows x cols,
src/vortex_container.h:55) when the wings share one shape.

Reference behaviour that is kept:

* the wake term of the solve is dropped (src/linear.inl:151, a discarded
  statement) unless `drop_wake_term=False`;
* only the first wing sheds wake (the reference's "TODO multiple wings");
* Katz-Plotkin loads see an empty UVLMVortexRing (simulator.cpp:37, 183), so
  their wake and chordwise-bound velocities are zero;
* the load row per wing is F / (0.5 rho U^2 S) with S = chord x span of the
  half-wing description, then Pin and Pout.
"""
from __future__ import annotations

import numpy as np

from . import Morphing, rings


class Wing:
    """proto::Wing (proto/uvlm.proto:11-30): the half-wing lattice (rows + 1) x (cols + 1) points at y >= 0,
    index j + i (cols + 1), plus origin, chord and span."""

    def __init__(self, rows: int, cols: int, points, origin=(0.0, 0.0, 0.0), chord: float = 1.0,
                 span: float = 1.0):
        self.rows, self.cols = int(rows), int(cols)
        self.points = np.asarray(points, dtype=np.float64).reshape(self.rows + 1, self.cols + 1, 3).copy()
        self.origin = np.asarray(origin, dtype=np.float64).reshape(3).copy()
        self.chord, self.span = float(chord), float(span)

    @classmethod
    def rect(cls, chord: float, span: float, rows: int, cols: int, origin=(0.0, 0.0, 0.0)) -> "Wing":
        """RectGenerator::Generate (src/wing/rect.cpp:18-44) with uniform spacing (WingGenerator::Generate,
        src/wing/wing_generator.h:18-26, stores chord, span, rows, cols)."""
        xs = np.linspace(0.0, chord, rows + 1)
        ys = np.linspace(0.0, span, cols + 1)
        X, Y = np.meshgrid(xs, ys, indexing="ij")
        return cls(rows, cols, np.stack([X, Y, np.zeros_like(X)], -1), origin, chord, span)


def transform_row(row: np.ndarray) -> np.ndarray:
    """internal::TransformRow (src/wing_builder.h:21-35): the mirrored points (reversed, y negated, without
    the root point) followed by the row itself."""
    row = np.asarray(row, dtype=np.float64)
    mirrored = row[1:][::-1].copy()
    mirrored[:, 1] *= -1
    return np.concatenate([mirrored, row])


def build_container_rings(wing: Wing) -> np.ndarray:
    """WingBuilder::AddWing + BuildWing (src/wing_builder.cpp:12-76): the full-span ring nodes
    (rows, 2 cols, 4, 3), ring (i, j) = points (i, j), (i+1, j), (i+1, j+1), (i, j+1), shifted by the origin."""
    pts = np.stack([transform_row(wing.points[i]) for i in range(wing.rows + 1)]) + wing.origin
    return np.stack([pts[:-1, :-1], pts[1:, :-1], pts[1:, 1:], pts[:-1, 1:]], axis=2)


class LegacySimulator:
    """UVLM::simulator::{AddWing, SetInlet, Start} (src/simulator/simulator.cpp:205-270) as an object."""

    def __init__(self, disable_wake: bool = False, use_joukowski: bool = False, drop_wake_term: bool = True):
        self.disable_wake = bool(disable_wake)
        self.use_joukowski = bool(use_joukowski)
        self.drop_wake_term = bool(drop_wake_term)
        self.wings: list[Wing] = []
        self.morphings: list[Morphing] = []
        self.inlet = np.array([1.0, 0.0, 0.0])
        self.output_path = ""
        self.output_load_path = ""

    def AddWing(self, wing: Wing, morphing: Morphing) -> None:  # noqa: N802 (reference name)
        """simulator::AddWing (simulator.cpp:205-209): the morphing takes the wing's origin."""
        m = Morphing()
        m.k = type(morphing.k).from_buffer_copy(morphing.k)
        m.set_origin(wing.origin)
        self.wings.append(wing)
        self.morphings.append(m)

    def SetInlet(self, x: float, y: float, z: float) -> None:  # noqa: N802
        self.inlet = np.array([x, y, z], dtype=np.float64)

    def SetOutputPath(self, path: str) -> None:  # noqa: N802
        """simulator::SetOutputPath (simulator.cpp:216): the directory of the per-step Snapshot2 files
        ("" writes none)."""
        self.output_path = str(path)

    def SetOutputLoadPath(self, path: str) -> None:  # noqa: N802
        """simulator::SetOutputLoadPath (simulator.cpp:218): the load file ("" writes none)."""
        self.output_load_path = str(path)

    # -- state -----------------------------------------------------------------
    def _create_containers(self) -> None:
        """CreateContainers (simulator.cpp:70-80): bound rings of every wing one after another."""
        if not self.wings:
            raise ValueError("No wing")
        blocks = [build_container_rings(w) for w in self.wings]
        self.shapes = [(b.shape[0], b.shape[1]) for b in blocks]
        self.sizes = [r * c for r, c in self.shapes]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(int)
        self.bound0 = np.concatenate([b.reshape(-1, 4, 3) for b in blocks])
        self.bound = self.bound0.copy()
        self.bound_gamma = np.zeros(len(self.bound))
        self.wake = np.zeros((0, 4, 3))
        self.wake0 = np.zeros((0, 4, 3))
        self.wake_gamma = np.zeros(0)

    def _edge(self):
        """Trailing-edge rings of the first wing (VortexContainer::edge_begin/end, vortex_container.h:128-131)."""
        rows, cols = self.shapes[0]
        return slice((rows - 1) * cols, rows * cols)

    def vortices(self):
        """The ring pool (bound rings, then wake rings) and its circulations."""
        return np.concatenate([self.bound, self.wake]), np.concatenate([self.bound_gamma, self.wake_gamma])

    def morphing_velocities(self, t: float):
        """The MorphingVelocity records of OutputSnapshot2 (simulator.cpp:135-152), one per bound ring:
        Morphing::Velocity at the reference centroid (VortexRing::ReferenceCentroid, src/vortex.cpp:102-104)
        and at (start0 + end0) / 2 of each segment in ForEachSegment order (src/vortex.h:149-160:
        start0 = nodes0[(q + 1) % 4], end0 = nodes0[q]), and the inlet.  Returns (center (n, 3),
        nodes (n, 4, 3), freestream (n, 3))."""
        b0 = self.bound0
        cent = (b0[:, 0] + b0[:, 1] + b0[:, 2] + b0[:, 3]) / 4
        mids = (np.roll(b0, -1, axis=1) + b0) / 2
        center = np.zeros_like(cent)
        nodes = np.zeros_like(mids)
        for c, m in enumerate(self.morphings):
            a, b = self.offsets[c], self.offsets[c + 1]
            v = m.Velocity(np.concatenate([cent[a:b], mids[a:b].reshape(-1, 3)]), t)
            center[a:b] = v[:b - a]
            nodes[a:b] = v[b - a:].reshape(-1, 4, 3)
        return center, nodes, np.tile(self.inlet, (len(b0), 1))

    def _output_snapshot2(self, step: int, t: float) -> None:
        """OutputSnapshot2 (simulator.cpp:118-160) to output_path/%08d."""
        import os

        from . import output

        pool, pool_g = self.vortices()
        pool0 = np.concatenate([self.bound0, self.wake0])
        center, nodes, fs = self.morphing_velocities(t)
        shapes = [(r, c, w.chord, w.span) for (r, c), w in zip(self.shapes, self.wings)]
        output.write_legacy_snapshot2(os.path.join(self.output_path, f"{step:08d}"), t, shapes, pool, pool0,
                                      pool_g, center, nodes, fs)

    def _morphing_process(self, t: float) -> None:
        """MorphingProcess + ConnectProcess (simulator.cpp:82-108)."""
        for c, m in enumerate(self.morphings):
            a, b = self.offsets[c], self.offsets[c + 1]
            self.bound[a:b] = m.Perfome(self.bound0[a:b].reshape(-1, 3), t).reshape(-1, 4, 3)
        e = self._edge()
        n_edge = e.stop - e.start
        if len(self.wake) >= n_edge:
            self.wake[:n_edge, 0] = self.bound[e, 1]
            self.wake[:n_edge, 3] = self.bound[e, 2]

    def _loads(self, t: float, dt: float, gamma_prev: np.ndarray) -> list[float]:
        """CalcLoadProcess (simulator.cpp:162-200)."""
        row = []
        pool, pool_g = self.vortices()
        rho = 1.0
        U = float(np.linalg.norm(self.inlet))
        for c, (w, m) in enumerate(zip(self.wings, self.morphings)):
            a, b = self.offsets[c], self.offsets[c + 1]
            rows, cols = self.shapes[c]
            if self.use_joukowski:
                load = rings.CalcLoadJoukowski(self.bound[a:b], self.bound0[a:b], self.bound_gamma[a:b],
                                               gamma_prev[a:b], rows, cols, m, pool, pool_g, self.inlet, rho, t, dt)
            else:
                load = rings.CalcLoadKatzPlotkin(self.bound[a:b], self.bound_gamma[a:b], gamma_prev[a:b], rows,
                                                 cols, m, self.inlet, rho, t, dt)
            S = w.chord * w.span
            coeff = load[:3] / (0.5 * rho * U * U * S)
            row += [float(coeff[0]), float(coeff[1]), float(coeff[2]), float(load[3]), float(load[4])]
        return row

    def Start(self, steps: int, dt: float) -> np.ndarray:  # noqa: N802
        """simulator::Start (simulator.cpp:220-270).  Returns one row per step: t, then per wing
        C_x, C_y, C_z, Pin, Pout (the load file's columns)."""
        self._create_containers()
        if self.output_load_path:
            open(self.output_load_path, "w").close()  # CheckReady (simulator.cpp:55-65) truncates it
        out = []
        for step in range(int(steps) + 1):
            t = dt * step
            gamma_prev = self.bound_gamma.copy()
            self._morphing_process(t)
            self.bound_gamma = rings.SolveLinearProblemContainers(
                self.bound, self.sizes, self.morphings, self.wake, self.wake_gamma, self.inlet, t,
                drop_wake_term=self.drop_wake_term, bound_rings0=self.bound0)
            if self.output_path:
                self._output_snapshot2(step, t)
            out.append([t] + self._loads(t, dt, gamma_prev))
            if self.output_load_path:
                with open(self.output_load_path, "a") as f:
                    f.write("\t".join(f"{v:g}" for v in out[-1]) + "\n")
            if step == steps:
                break
            if not self.disable_wake:
                e = self._edge()
                wake_next = np.concatenate([self.bound[e], self.wake])
                wake_next_gamma = np.concatenate([self.bound_gamma[e], self.wake_gamma])
                pool, pool_g = self.vortices()
                self.wake = rings.AdvectParallel(pool, pool_g, wake_next, self.inlet, dt)
                self.wake0 = np.concatenate([self.bound0[e], self.wake0])  # shed rings keep the edge's nodes0
                self.wake_gamma = wake_next_gamma
        return np.array(out)
