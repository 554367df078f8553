"""The inputs of the reference's fast marching examples
(examples/serial/fast_marching_method/*.c), restated in numpy with the same
arithmetic.  Arrays are C-ordered (ny, nx) or (nz, ny, nx), x fastest as in
the examples; spacing is in x, y(, z) order."""
import numpy as np


def _axis(n, lo=-1.0, hi=1.0):
    dx = (hi - lo) / n
    return lo + dx * np.arange(n + 1), dx


def distance_3d():
    """computeDistanceFunction3d.c:57-82: a sphere of radius 0.5 on [-1, 1]^3,
    51 points per axis, phi = |x|^2 - r^2, order 2."""
    a, dx = _axis(50)
    z, y, x = np.meshgrid(a, a, a, indexing="ij")
    phi = (x - 0.0) * (x - 0.0) + (y - 0.0) * (y - 0.0) + (z - 0.0) * (z - 0.0) - 0.5 * 0.5
    return np.ascontiguousarray(phi), [dx, dx, dx]


def distance_2d():
    """computeDistanceFunction2d.c:57-79: a circle of radius 0.5 on
    [-1, 1]^2, 101 points per axis, order 2."""
    a, dx = _axis(100)
    y, x = np.meshgrid(a, a, indexing="ij")
    phi = (x - 0.0) * (x - 0.0) + (y - 0.0) * (y - 0.0) - 0.5 * 0.5
    return np.ascontiguousarray(phi), [dx, dx]


def extension_2d():
    """computeExtensionFields2d.c:62-109: two circles of radius 0.2 at
    (0.25, 0.25) and (-0.25, -0.25), 64 points per axis, signed distances;
    sources sin((k+1) x) + cos((2k+1) y), k = 0, 1; order 2."""
    a, dx = _axis(63)
    y, x = np.meshgrid(a, a, indexing="ij")
    d1 = np.sqrt((x - 0.25) * (x - 0.25) + (y - 0.25) * (y - 0.25)) - 0.2
    d2 = np.sqrt((x + 0.25) * (x + 0.25) + (y + 0.25) * (y + 0.25)) - 0.2
    phi = np.where(d1 < d2, d1, d2)
    src = [np.ascontiguousarray(np.sin((k + 1) * x) + np.cos((2 * k + 1) * y))
           for k in range(2)]
    return np.ascontiguousarray(phi), src, [dx, dx]


def eikonal_2d():
    """solveEikonalEquation2d.c:57-92: phi = 0 inside the circle of radius
    0.5 (the boundary data) and -1 outside, speed 1 for x < 0 and 2 else,
    101 points per axis, order 2."""
    a, dx = _axis(100)
    y, x = np.meshgrid(a, a, indexing="ij")
    inside = (x - 0.0) * (x - 0.0) + (y - 0.0) * (y - 0.0) - 0.5 * 0.5 < 0
    phi = np.where(inside, 0.0, -1.0)
    speed = np.where(x < 0, 1.0, 2.0)
    return np.ascontiguousarray(phi), np.ascontiguousarray(speed), [dx, dx]
