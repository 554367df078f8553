"""Signed distance functions, extension fields and Eikonal solutions on the
GPU (the reference pylsmlib's ``computeDistanceFunction``,
``computeExtensionFields``, ``solveEikonalEquation`` and ``travel_time``,
pylsmlib/pylsmlib/__init__.py:27-183, lsmlib.pyx:10-120).

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


def computeExtensionFields(phi0, speed, dx=1.0, order=2, mask=None, ext_mask=None):
    """(distance function, extension fields): ``speed`` of phi0's shape or
    (N,) + phi0.shape, extended off the zero level set of phi0 as the
    reference does (computeExtensionFields3d).  ``ext_mask`` is boolean:
    True marks the points whose own source value is used at the interface
    (the reference passes it on as -ext_mask * 2 + 1)."""
    phi = np.ascontiguousarray(np.asarray(phi0, dtype=np.float64))
    if phi.ndim not in (1, 2, 3):
        raise ValueError("phi0 must be 1D, 2D or 3D")
    dims, spacing = _dims_dx(phi.shape, dx)
    if order not in (1, 2):
        raise ValueError("order must be 1 or 2")
    u0 = np.asarray(speed, dtype=np.float64)
    u0shape = u0.shape
    if u0shape == phi.shape:
        u0 = u0.reshape((1,) + u0shape)
    if u0.shape[1:] != phi.shape:
        raise ValueError("phi and speed must have the same shape")
    m = None
    if mask is not None:
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.float64))
        if m.shape != phi.shape:
            raise ValueError("phi and mask have incompatible shapes")
    em = None
    if ext_mask is not None:
        em = np.asarray(ext_mask, dtype=np.float64)
        if em.shape != phi.shape:
            raise ValueError("phi and extensionMask have incompatible shapes")
        em = np.ascontiguousarray(-em * 2.0 + 1.0)
    nf = u0.shape[0]
    src = [np.ascontiguousarray(u0[k]) for k in range(nf)]
    ext = [np.empty_like(phi) for _ in range(nf)]
    dist = np.empty_like(phi)
    lib = gpu.load()
    gd = (ctypes.c_int * 3)(*dims)
    h = (ctypes.c_double * 3)(*spacing)
    src_p = (ctypes.c_void_p * max(nf, 1))(*[a.ctypes.data for a in src])
    ext_p = (ctypes.c_void_p * max(nf, 1))(*[a.ctypes.data for a in ext])
    rc = lib.lsmgpu_extension_fields3d(dist.ctypes.data, ctypes.cast(ext_p, ctypes.c_void_p),
                                       phi.ctypes.data, None if m is None else m.ctypes.data,
                                       ctypes.cast(src_p, ctypes.c_void_p),
                                       None if em is None else em.ctypes.data, nf, int(order),
                                       gd, h, None)
    gpu.check_rc(rc, "extension_fields3d")
    return dist, np.stack(ext).reshape(u0shape)


def solveEikonalEquation(phi0, speed, dx=1.0, order=2):
    """phi with |grad phi| speed = 1 and phi = 0 where phi0 = 0, as the
    reference's Python wrapper computes it: the region phi0 <= 0 (shifted
    by -min(phi0)) is the boundary data, the rest is solved for
    (solveEikonalEquation3d), and the shift is undone (lsmlib.pyx:98-120)."""
    phi = np.array(np.asarray(phi0, dtype=np.float64), order="C", copy=True)
    if phi.ndim not in (1, 2, 3):
        raise ValueError("phi0 must be 1D, 2D or 3D")
    dims, spacing = _dims_dx(phi.shape, dx)
    if order not in (1, 2):
        raise ValueError("order must be 1 or 2")
    f = np.ascontiguousarray(np.asarray(speed, dtype=np.float64))
    if f.shape != phi.shape:
        raise ValueError("phi and speed must have the same shape")
    minphi = phi.min()
    phi[phi > 0] = minphi - 1.0
    phi -= minphi
    lib = gpu.load()
    gd = (ctypes.c_int * 3)(*dims)
    h = (ctypes.c_double * 3)(*spacing)
    rc = lib.lsmgpu_eikonal3d(phi.ctypes.data, f.ctypes.data, None, int(order), gd, h, None)
    gpu.check_rc(rc, "eikonal3d")
    phi += minphi
    return phi


def travel_time(phi0, speed, dx=1.0, order=2):
    """|solveEikonalEquation(phi0, speed, dx, order)|."""
    return abs(solveEikonalEquation(phi0, speed, dx, order))
