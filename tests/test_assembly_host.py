"""The algebra of the unique-segment influence matrix (no GPU).

The assembly kernels (step.cu / batch.cu `assemble_kernel`, `b_assemble_kernel`)
combine, for ring (i, j) of a lattice, the spanwise segment S(i, j) = (i, j) ->
(i, j+1) and the chordwise H(i, j+1) = (i, j+1) -> (i+1, j+1) forwards with
S(i+1, j) and H(i, j) backwards, each segment evaluated once per collocation
point and shared by its two rings.  This checks that combination, in FP64
numpy, against VORING's four segments p0 -> p1 -> p2 -> p3 -> p0
(src/vortex.cpp:145-160) with the reference's segment law and cut-offs
(src/vortex.cpp:21-39), on random lattices and at the rings' own centroids.
"""
import numpy as np

CUT = 1e-10


def segment(x, a, b):
    """Biot-Savart velocity of the unit segment a -> b at the points x (N, 3)."""
    r1, r2 = x - a, x - b
    r0 = b - a
    d = np.cross(r1, r2)
    d2 = np.einsum("ij,ij->i", d, d)
    n1, n2 = np.linalg.norm(r1, axis=1), np.linalg.norm(r2, axis=1)
    ok = (d2 >= CUT) & (n1 >= CUT) & (n2 >= CUT)
    with np.errstate(divide="ignore", invalid="ignore"):
        k = np.einsum("j,ij->i", r0, r1 / n1[:, None] - r2 / n2[:, None]) / (4 * np.pi * d2)
    return np.where(ok[:, None], d * k[:, None], 0.0)


def ring_form(x, p):
    R, C = p.shape[0] - 1, p.shape[1] - 1
    out = np.zeros((x.shape[0], R, C, 3))
    for i in range(R):
        for j in range(C):
            q = [p[i, j], p[i, j + 1], p[i + 1, j + 1], p[i + 1, j]]
            for s in range(4):
                out[:, i, j] += segment(x, q[s], q[(s + 1) % 4])
    return out


def unique_segment_form(x, p):
    R, C = p.shape[0] - 1, p.shape[1] - 1
    S = np.zeros((x.shape[0], R + 1, C, 3))   # (i, j) -> (i, j+1)
    H = np.zeros((x.shape[0], R, C + 1, 3))   # (i, j) -> (i+1, j)
    for i in range(R + 1):
        for j in range(C):
            S[:, i, j] = segment(x, p[i, j], p[i, j + 1])
    for i in range(R):
        for j in range(C + 1):
            H[:, i, j] = segment(x, p[i, j], p[i + 1, j])
    return S[:, :-1] + H[:, :, 1:] - S[:, 1:] - H[:, :, :-1]


def test_unique_segments_reproduce_the_ring_form():
    rng = np.random.default_rng(7)
    for R, C in [(1, 1), (3, 5), (4, 8), (6, 3)]:
        ii, jj = np.meshgrid(np.arange(R + 1), np.arange(C + 1), indexing="ij")
        p = np.stack([0.3 * ii, 0.5 * jj, 0.05 * np.sin(ii + 2 * jj)], axis=-1)
        p = p + 0.02 * rng.standard_normal(p.shape)
        # the rings' centroids (collocation points), random points, and two nodes (cut pairs)
        cen = 0.25 * (p[:-1, :-1] + p[:-1, 1:] + p[1:, 1:] + p[1:, :-1]).reshape(-1, 3)
        x = np.concatenate([cen, rng.uniform(-1, 4, (20, 3)), p[0, :1], p[R, C:]])
        a = ring_form(x, p)
        b = unique_segment_form(x, p)
        scale = np.abs(a).max()
        assert np.abs(a - b).max() <= 1e-13 * scale


def test_backward_segment_is_the_negated_forward_one():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((50, 3))
    a, b = rng.standard_normal(3), rng.standard_normal(3)
    np.testing.assert_allclose(segment(x, b, a), -segment(x, a, b), rtol=1e-13, atol=1e-15)
