"""Signed distance functions on the GPU (the reference pylsmlib's
``computeDistanceFunction``, pylsmlib/pylsmlib/__init__.py:27-84).

``computeDistanceFunction(phi0, dx, order)`` returns the distance function of
the zero level set of ``phi0`` with the values of the reference's fast
marching method (first- or second-order update), computed by
lsmgpu_distance_function3d in liblsmgpu.so.  As in the reference, the array
shape gives the dimension and the layout is C order: (nx,), (ny, nx) or
(nz, ny, nx), with ``dx`` per axis in the same order (a scalar is used for
every axis), and the same ValueErrors for a bad dx or order.  The
reference's Python package stops at 2D; 3D is supported here, and ``mask``
(< 0 marks points outside the domain, which get LSMLIB_REAL_MAX) is passed
through as the C routine takes it.
"""
import ctypes

import numpy as np

from lsmlib_b200 import gpu


def _dims_dx(shape, dx):
    """(nx, ny, nz) and (dx, dy, dz) for an array of ``shape`` (C order)."""
    d = np.atleast_1d(np.asarray(dx, dtype=np.float64))
    if d.size == 1:
        d = np.repeat(d, len(shape))
    if d.size != len(shape):
        raise ValueError("dx must be of length len(phi.shape)")
    if np.prod(d) == 0:
        raise ValueError("dx must be greater than zero")
    dims = list(reversed(shape)) + [1] * (3 - len(shape))
    spacing = list(reversed(d.tolist())) + [1.0] * (3 - len(shape))
    return dims, spacing


def computeDistanceFunction(phi0, dx=1.0, order=2, mask=None):
    """Distance function of the zero level set of phi0 (numpy in, numpy out)."""
    phi = np.ascontiguousarray(np.asarray(phi0, dtype=np.float64))
    if phi.ndim not in (1, 2, 3):
        raise ValueError("phi0 must be 1D, 2D or 3D")
    dims, spacing = _dims_dx(phi.shape, dx)
    if order not in (1, 2):
        raise ValueError("order must be 1 or 2")
    m = None
    if mask is not None:
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.float64))
        if m.shape != phi.shape:
            raise ValueError("mask must have the shape of phi0")
    out = np.empty_like(phi)
    lib = gpu.load()
    gd = (ctypes.c_int * 3)(*dims)
    h = (ctypes.c_double * 3)(*spacing)
    rc = lib.lsmgpu_distance_function3d(out.ctypes.data, phi.ctypes.data,
                                        None if m is None else m.ctypes.data, int(order),
                                        gd, h, None)
    gpu.check_rc(rc, "distance_function3d")
    return out
