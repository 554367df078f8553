"""Argument checks of the fast marching entry points through the C ABI.

Every check runs before the first CUDA call, so these tests need no GPU.
The reference's names keep its return codes: 2 for an order other than 1 or
2, and -1 for any other failure (src/serial/lsm_fast_marching_method.h:
331-341, 386-392, 463-469). The lsmgpu_ names return the library's status
codes and record a message."""
import ctypes

import numpy as np
import pytest

from lsmlib_b200 import gpu

P = ctypes.c_void_p
SUCCESS, INVALID_BOX, NULL_POINTER, INVALID_VALUE = 0, 1, 2, 5


@pytest.fixture(scope="module")
def lib():
    lib = gpu.load()
    lib.computeDistanceFunction3d.argtypes = [P] * 3 + [ctypes.c_int, P, P]
    lib.computeExtensionFields3d.argtypes = [P] * 6 + [ctypes.c_int, ctypes.c_int, P, P]
    lib.solveEikonalEquation3d.argtypes = [P] * 3 + [ctypes.c_int, P, P]
    for f in ("computeDistanceFunction3d", "computeExtensionFields3d",
              "solveEikonalEquation3d"):
        getattr(lib, f).restype = ctypes.c_int
    return lib


def arrays(dims=(4, 5, 6), dx=(1.0, 1.0, 1.0)):
    phi = np.zeros(dims[::-1])
    return (phi, np.zeros_like(phi), np.array(dims, dtype=np.intc),
            np.array(dx, dtype=np.float64))


def message(lib):
    return lib.lsmgpu_get_last_error_string().decode()


def distance(lib, out, phi, order, dims, dx):
    return lib.lsmgpu_distance_function3d(
        None if out is None else out.ctypes.data, None if phi is None else phi.ctypes.data,
        None, order, dims.ctypes.data, dx.ctypes.data, None)


def test_distance_rejects_bad_order(lib):
    phi, out, dims, dx = arrays()
    for order in (0, 3, -1):
        assert lib.computeDistanceFunction3d(out.ctypes.data, phi.ctypes.data, None, order,
                                             dims.ctypes.data, dx.ctypes.data) == 2
        assert distance(lib, out, phi, order, dims, dx) == INVALID_VALUE
        assert "order" in message(lib)


def test_distance_rejects_null_arrays(lib):
    phi, out, dims, dx = arrays()
    assert lib.computeDistanceFunction3d(None, phi.ctypes.data, None, 1, dims.ctypes.data,
                                         dx.ctypes.data) == -1
    assert distance(lib, out, None, 1, dims, dx) == NULL_POINTER
    assert "null" in message(lib)
    assert lib.lsmgpu_distance_function3d(out.ctypes.data, phi.ctypes.data, None, 1, None,
                                          dx.ctypes.data, None) == NULL_POINTER


@pytest.mark.parametrize("dims", [(0, 5, 6), (4, -1, 6), (4, 5, 0)])
def test_distance_rejects_empty_grid(lib, dims):
    phi, out, _, dx = arrays()
    d = np.array(dims, dtype=np.intc)
    assert distance(lib, out, phi, 2, d, dx) == INVALID_BOX
    assert "empty grid" in message(lib)


@pytest.mark.parametrize("h", [(0.0, 1.0, 1.0), (1.0, -0.5, 1.0), (1.0, 1.0, np.inf),
                               (np.nan, 1.0, 1.0)])
def test_distance_rejects_bad_spacing(lib, h):
    phi, out, dims, _ = arrays()
    assert distance(lib, out, phi, 1, dims, np.array(h)) == INVALID_VALUE
    assert "dx" in message(lib)


def test_distance_rejects_more_than_2_31_points(lib):
    """The point lists hold 32-bit indices; a 2048 x 2048 x 1024 grid is
    refused before any array is read (the arrays here are small stand-ins)."""
    phi, out, _, dx = arrays()
    d = np.array([2048, 2048, 1024], dtype=np.intc)
    assert distance(lib, out, phi, 1, d, dx) == INVALID_BOX
    assert "2^31" in message(lib)


def test_extension_rejects_bad_field_arguments(lib):
    phi, out, dims, dx = arrays()
    src = np.zeros_like(phi)
    ext_p = (ctypes.c_void_p * 1)(None)
    src_p = (ctypes.c_void_p * 1)(src.ctypes.data)
    rc = lib.lsmgpu_extension_fields3d(out.ctypes.data, ctypes.cast(ext_p, P), phi.ctypes.data,
                                       None, ctypes.cast(src_p, P), None, 1, 1,
                                       dims.ctypes.data, dx.ctypes.data, None)
    assert rc == NULL_POINTER and "field" in message(lib)
    rc = lib.lsmgpu_extension_fields3d(out.ctypes.data, None, phi.ctypes.data, None, None,
                                       None, -1, 1, dims.ctypes.data, dx.ctypes.data, None)
    assert rc == INVALID_VALUE and "field count" in message(lib)
    assert lib.computeExtensionFields3d(out.ctypes.data, None, phi.ctypes.data, None, None,
                                        None, 0, 5, dims.ctypes.data, dx.ctypes.data) == 2


def test_eikonal_rejects_bad_arguments(lib):
    phi, speed, dims, dx = arrays()
    assert lib.solveEikonalEquation3d(phi.ctypes.data, speed.ctypes.data, None, 4,
                                      dims.ctypes.data, dx.ctypes.data) == 2
    assert lib.solveEikonalEquation3d(phi.ctypes.data, None, None, 1, dims.ctypes.data,
                                      dx.ctypes.data) == -1
    assert lib.lsmgpu_eikonal3d(phi.ctypes.data, None, None, 1, dims.ctypes.data,
                                dx.ctypes.data, None) == NULL_POINTER
    bad = np.array([1.0, 0.0, 1.0])
    assert lib.lsmgpu_eikonal3d(phi.ctypes.data, speed.ctypes.data, None, 2,
                                dims.ctypes.data, bad.ctypes.data, None) == INVALID_VALUE
    d = np.array([2048, 2048, 1024], dtype=np.intc)
    assert lib.lsmgpu_eikonal3d(phi.ctypes.data, speed.ctypes.data, None, 1, d.ctypes.data,
                                dx.ctypes.data, None) == INVALID_BOX


def test_2d_entry_points_check_arguments(lib):
    """The 2D forms (lsm_fast_marching_method.h:124-134, 179-185, 256-262)
    keep the reference's return codes: 2 for a bad order, -1 otherwise."""
    phi = np.zeros((5, 4))
    out = np.zeros_like(phi)
    dims = np.array([4, 5], dtype=np.intc)
    dx = np.array([1.0, 1.0])
    f = lib.computeDistanceFunction2d
    f.argtypes, f.restype = [P] * 3 + [ctypes.c_int, P, P], ctypes.c_int
    assert f(out.ctypes.data, phi.ctypes.data, None, 3, dims.ctypes.data, dx.ctypes.data) == 2
    assert f(out.ctypes.data, None, None, 1, dims.ctypes.data, dx.ctypes.data) == -1
    assert f(out.ctypes.data, phi.ctypes.data, None, 1, None, dx.ctypes.data) == -1
    assert f(out.ctypes.data, phi.ctypes.data, None, 1, dims.ctypes.data, None) == -1
    bad = np.array([1.0, -1.0])
    assert f(out.ctypes.data, phi.ctypes.data, None, 2, dims.ctypes.data, bad.ctypes.data) == -1
    assert "dx" in message(lib)
    g = lib.computeExtensionFields2d
    g.argtypes, g.restype = [P] * 6 + [ctypes.c_int, ctypes.c_int, P, P], ctypes.c_int
    assert g(out.ctypes.data, None, phi.ctypes.data, None, None, None, 0, 0,
             dims.ctypes.data, dx.ctypes.data) == 2
    assert g(out.ctypes.data, None, phi.ctypes.data, None, None, None, -2, 1,
             dims.ctypes.data, dx.ctypes.data) == -1
    e = lib.solveEikonalEquation2d
    e.argtypes, e.restype = [P] * 3 + [ctypes.c_int, P, P], ctypes.c_int
    assert e(phi.ctypes.data, phi.ctypes.data, None, 5, dims.ctypes.data, dx.ctypes.data) == 2
    assert e(phi.ctypes.data, None, None, 1, dims.ctypes.data, dx.ctypes.data) == -1
