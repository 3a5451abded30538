"""The reference's legacy stepper (src/simulator/simulator.{h,cpp}) over AoS vortex rings.

The legacy API keeps every ring of every wing and of the wake in one pool of
`VortexRing`s (src/vortex_container.h:22-136); a `VortexContainer` is a
rows x cols view of a wing's bound rings in it.  `LegacySimulator.Start`
runs the legacy main loop (simulator.cpp:220-270): Morphing of the bound
rings and reconnection of the newest wake row to the trailing edge
(:82-108), the circulation solve of linear.inl (:110-116), the loads of the
chosen formulation (:162-200), then shedding and roll-up of the wake by
AdvectParallel (:252-266).  Each stage is one call of the C-ABI (the CUDA
kernels); the host only moves the AoS arrays.  Per-step Snapshot2 output
(:118-160) is not written.

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

    def AddWing(self, wing: Wing, morphing: Morphing) -> None:  # noqa: N802 (reference name)
        """simulator::AddWing (simulator.cpp:205-209): the morphing takes the wing's origin."""
        m = Morphing()
        m.k = type(morphing.k).from_buffer_copy(morphing.k)
        m.set_origin(wing.origin)
        self.wings.append(wing)
        self.morphings.append(m)

    def SetInlet(self, x: float, y: float, z: float) -> None:  # noqa: N802
        self.inlet = np.array([x, y, z], dtype=np.float64)

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
        self.wake_gamma = np.zeros(0)

    def _edge(self):
        """Trailing-edge rings of the first wing (VortexContainer::edge_begin/end, vortex_container.h:128-131)."""
        rows, cols = self.shapes[0]
        return slice((rows - 1) * cols, rows * cols)

    def vortices(self):
        """The ring pool (bound rings, then wake rings) and its circulations."""
        return np.concatenate([self.bound, self.wake]), np.concatenate([self.bound_gamma, self.wake_gamma])

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
        out = []
        for step in range(int(steps) + 1):
            t = dt * step
            gamma_prev = self.bound_gamma.copy()
            self._morphing_process(t)
            self.bound_gamma = rings.SolveLinearProblemContainers(
                self.bound, self.sizes, self.morphings, self.wake, self.wake_gamma, self.inlet, t,
                drop_wake_term=self.drop_wake_term, bound_rings0=self.bound0)
            out.append([t] + self._loads(t, dt, gamma_prev))
            if step == steps:
                break
            if not self.disable_wake:
                e = self._edge()
                wake_next = np.concatenate([self.bound[e], self.wake])
                wake_next_gamma = np.concatenate([self.bound_gamma[e], self.wake_gamma])
                pool, pool_g = self.vortices()
                self.wake = rings.AdvectParallel(pool, pool_g, wake_next, self.inlet, dt)
                self.wake_gamma = wake_next_gamma
        return np.array(out)
