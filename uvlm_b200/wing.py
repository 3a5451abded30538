"""Wing lattice generators (src/wing/*): host-side set-up of a wing's nodes.

A generator fills the node lattice of one half wing (chord x half span,
rows x half cols rings); ``WholeWing`` mirrors it into the whole wing in the
reference's node order.  ``SimpleSimulator.AddWing`` takes any generator, as
the reference's AddWing takes any ``wing::WingGenerator*``
(src/simulator/simple_simulator.h:50-53): a ``RectGenerator`` wing is built by
the library itself, any other generator's lattice is passed through
``uvlm_add_wing_nodes``.

  WingGenerator        src/wing/wing_generator.h:12-32
  RectGenerator        src/wing/rect.{h,cpp} (linspace or Chebyshev spacing)
  NACA4digitGenerator  src/wing/naca4digit.{h,cpp} (mean camber line)
  NACA00XXGenerator    src/wing/naca00XX.{h,cpp} (half thickness)
  WholeWing            src/wing/wing.cpp:12-52
"""
from __future__ import annotations

import math

import numpy as np


def linspace(a: float, b: float, n: int) -> np.ndarray:
    """util.h:36-43: a + i (b - a)/(n - 1), evaluated as the reference does."""
    dx = (b - a) / (n - 1)
    return np.array([a + i * dx for i in range(n)])


def transform_chebyshev(n: int, xmin: float, xmax: float) -> np.ndarray:
    """TransformChebyshev (src/wing/rect.h:16-25)."""
    th = linspace(-math.pi / 2, 0.0, n)
    r = np.array([xmin + (xmax - xmin) * math.cos(t) for t in th])
    r[0], r[-1] = xmin, xmax
    return r


def NACA4digit(x: float, c: float, xx: int) -> float:  # noqa: N802 (reference name)
    """Mean camber of a 4-digit NACA section at x for chord c (src/wing/naca4digit.cpp:12-27): only the
    first two digits matter, m = first/100 (maximum camber), p = second/10 (its position)."""
    first, second = xx // 10, xx % 10
    m, p = first / 100.0, second / 10.0
    if 0 <= x <= p * c:
        return m * x / p / p * (2 * p - x / c)
    if p * c <= x <= c:
        return m * (c - x) / (1 - p) / (1 - p) * (1 + x / c - 2 * p)
    return 0.0


def NACA00XX(x: float, c: float, xx: int) -> float:  # noqa: N802 (reference name)
    """Half thickness of a symmetric 4-digit NACA section (src/wing/naca00XX.cpp:14-19)."""
    t = xx * 0.01
    z = x / c
    return 5 * t * c * (0.2969 * math.sqrt(z) + (-0.1260) * (z) + (-0.3516) * z * z + 0.2843 * z * z * z +
                        (-0.1015) * z * z * z * z)


class WingGenerator:
    """Base of the lattice generators (src/wing/wing_generator.h:12-32)."""

    def Generate(self, chord: float, span: float, rows: int, cols: int) -> np.ndarray:  # noqa: N802
        """Node lattice of a (half) wing: (rows + 1, cols + 1, 3)."""
        raise NotImplementedError

    __call__ = Generate


class RectGenerator(WingGenerator):
    """Flat rectangular lattice (src/wing/rect.cpp:18-45): x = linspace(0, chord, rows + 1),
    y = linspace(0, span, cols + 1), z = 0, or Chebyshev spacing where chosen (the reference's
    --chebyshev_chord / --chebyshev_span flags)."""

    def __init__(self, chebyshev_chord: bool = False, chebyshev_span: bool = False):
        self.chebyshev_chord = bool(chebyshev_chord)
        self.chebyshev_span = bool(chebyshev_span)

    def Generate(self, chord, span, rows, cols):  # noqa: N802
        xs = transform_chebyshev(rows + 1, 0, chord) if self.chebyshev_chord else linspace(0, chord, rows + 1)
        ys = transform_chebyshev(cols + 1, 0, span) if self.chebyshev_span else linspace(0, span, cols + 1)
        pts = np.zeros((rows + 1, cols + 1, 3))
        pts[..., 0] = xs[:, None]
        pts[..., 1] = ys[None, :]
        return pts


class NACA4digitGenerator(RectGenerator):
    """Rectangular lattice with z = NACA4digit(x, chord, digit) (src/wing/naca4digit.cpp:29-39)."""

    def __init__(self, digit: int, chebyshev_chord: bool = False, chebyshev_span: bool = False):
        super().__init__(chebyshev_chord, chebyshev_span)
        self.digit = int(digit)

    def Generate(self, chord, span, rows, cols):  # noqa: N802
        pts = super().Generate(chord, span, rows, cols)
        pts[..., 2] = [[NACA4digit(x, chord, self.digit) for x in row] for row in pts[..., 0]]
        return pts


class NACA00XXGenerator(RectGenerator):
    """Rectangular lattice with z = NACA00XX(x, chord, digit) (src/wing/naca00XX.cpp:21-32)."""

    def __init__(self, digit: int, chebyshev_chord: bool = False, chebyshev_span: bool = False):
        super().__init__(chebyshev_chord, chebyshev_span)
        self.digit = int(digit)

    def Generate(self, chord, span, rows, cols):  # noqa: N802
        pts = super().Generate(chord, span, rows, cols)
        pts[..., 2] = [[NACA00XX(x, chord, self.digit) for x in row] for row in pts[..., 0]]
        return pts


def WholeWing(half: np.ndarray, origin=(0.0, 0.0, 0.0)) -> np.ndarray:  # noqa: N802 (reference name)
    """src/wing/wing.cpp:12-52: per node row, the mirror image (y -> -y) of the half row in reverse order,
    then the half row without its first node; finally + origin.  (rows + 1, 2 half_cols + 1, 3)."""
    half = np.asarray(half, dtype=np.float64)
    mirror = half.copy()
    mirror[..., 1] *= -1
    whole = np.concatenate([mirror[:, ::-1], half[:, 1:]], axis=1)
    return whole + np.asarray(origin, dtype=np.float64)
