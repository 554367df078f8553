"""Fast marching checks that reach beyond the 3D entry points: the 2D entry
points against the reference's golden outputs, and the reference Python
package's own known-answer doctests through pylsmlib.  Kept in a file of
their own, collected after the other GPU parity tests."""
import ctypes

import numpy as np
import pytest

from test_fmm_golden import GOLDEN, _case, eik_case, ext_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from lsmlib_b200 import gpu
    return gpu.load()


def same_bits(a, b):
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_2d_entry_points_reproduce_reference_golden(lib):
    """computeDistanceFunction2d, computeExtensionFields2d and
    solveEikonalEquation2d on the 2D golden case (grid_dims and dx in x, y).
    The golden outputs come from the reference's 3D routines on the same
    plane, which its 2D routines match bit for bit (test_fmm_golden.py), so
    bit-equality here is parity with the reference's 2D routines."""
    z = np.load(GOLDEN)
    phi3, dx3, _ = _case(z, "spheres2d")
    phi = np.ascontiguousarray(phi3[0])
    ny, nx = phi.shape
    P = ctypes.c_void_p
    dims = np.array([nx, ny], dtype=np.intc)
    h = np.array(dx3[:2], dtype=np.float64)
    dist_fn = lib.computeDistanceFunction2d
    dist_fn.argtypes, dist_fn.restype = [P] * 3 + [ctypes.c_int, P, P], ctypes.c_int
    ext_fn = lib.computeExtensionFields2d
    ext_fn.argtypes = [P] * 6 + [ctypes.c_int, ctypes.c_int, P, P]
    ext_fn.restype = ctypes.c_int
    eik_fn = lib.solveEikonalEquation2d
    eik_fn.argtypes, eik_fn.restype = [P] * 3 + [ctypes.c_int, P, P], ctypes.c_int
    src3, _ = ext_case(z, "spheres2d")
    src = [np.ascontiguousarray(s[0]) for s in src3]
    data3, speed3, _ = eik_case(z, "spheres2d")
    for order in (1, 2):
        out = np.full_like(phi, np.nan)
        assert dist_fn(out.ctypes.data, phi.ctypes.data, None, order, dims.ctypes.data,
                       h.ctypes.data) == 0
        assert same_bits(out, z["spheres2d|out%d" % order][0])
        dist = np.full_like(phi, np.nan)
        ext = [np.full_like(phi, np.nan) for _ in src]
        ext_p = (P * 2)(*[e.ctypes.data for e in ext])
        src_p = (P * 2)(*[s.ctypes.data for s in src])
        assert ext_fn(dist.ctypes.data, ctypes.cast(ext_p, P), phi.ctypes.data, None,
                      ctypes.cast(src_p, P), None, 2, order, dims.ctypes.data,
                      h.ctypes.data) == 0
        assert same_bits(dist, z["spheres2d|out%d" % order][0])
        for k in range(2):
            assert same_bits(ext[k], z["spheres2d|ext%d_%d" % (order, k)][0])
        sol = np.ascontiguousarray(data3[0]).copy()
        speed = np.ascontiguousarray(speed3[0])
        assert eik_fn(sol.ctypes.data, speed.ctypes.data, None, order, dims.ctypes.data,
                      h.ctypes.data) == 0
        assert same_bits(sol, z["spheres2d|eik%d" % order][0])


# ---- the reference package's own known-answer doctests, through pylsmlib ---------

from fmm_reference_cases import CASES as REFERENCE_CASES  # noqa: E402


class PylsmlibBackend:
    """pylsmlib's front door on the GPU, in the reference package's calls."""

    @staticmethod
    def distance(phi, dx, order):
        from pylsmlib import computeDistanceFunction
        return computeDistanceFunction(phi, dx=dx, order=order)

    @staticmethod
    def extension(phi, speed, dx, order, ext_mask):
        from pylsmlib import computeExtensionFields
        return computeExtensionFields(phi, speed, dx=dx, order=order, ext_mask=ext_mask)

    @staticmethod
    def travel_time(phi, speed, dx, order):
        from pylsmlib import travel_time
        return travel_time(phi, speed, dx, order)


@pytest.mark.parametrize("case", REFERENCE_CASES, ids=[c.__name__ for c in REFERENCE_CASES])
def test_pylsmlib_reference_doctest_case(case):
    """pylsmlib/pylsmlib/__init__.py:196-800; the same cases pass on the
    reference's own routines and on the oracle (test_fmm_reference_doctests.py)."""
    case(PylsmlibBackend())


# ---- the reference's fast marching examples, through the C entry points ------------

import fmm_example_cases as examples  # noqa: E402
import oracle  # noqa: E402


def test_reference_examples_match_oracle(lib):
    """The inputs of examples/serial/fast_marching_method/*.c through the
    entry points each example calls (computeDistanceFunction3d and the 2D
    forms), on host arrays, bit for bit against the oracle (one plane thick
    for 2D)."""
    P = ctypes.c_void_p
    f3 = lib.computeDistanceFunction3d
    f2 = lib.computeDistanceFunction2d
    for f in (f3, f2):
        f.argtypes, f.restype = [P] * 3 + [ctypes.c_int, P, P], ctypes.c_int
    e2 = lib.computeExtensionFields2d
    e2.argtypes, e2.restype = [P] * 6 + [ctypes.c_int, ctypes.c_int, P, P], ctypes.c_int
    k2 = lib.solveEikonalEquation2d
    k2.argtypes, k2.restype = [P] * 3 + [ctypes.c_int, P, P], ctypes.c_int

    def grid(phi, dx):
        return np.array(phi.shape[::-1], dtype=np.intc), np.array(dx, dtype=np.float64)

    phi, dx = examples.distance_3d()
    out = np.full_like(phi, np.nan)
    d, h = grid(phi, dx)
    assert f3(out.ctypes.data, phi.ctypes.data, None, 2, d.ctypes.data, h.ctypes.data) == 0
    assert same_bits(out, oracle.oracle_fmm(ordered=True)(phi, 2, dx))
    phi, dx = examples.distance_2d()
    out = np.full_like(phi, np.nan)
    d, h = grid(phi, dx)
    assert f2(out.ctypes.data, phi.ctypes.data, None, 2, d.ctypes.data, h.ctypes.data) == 0
    assert same_bits(out, oracle.oracle_fmm(ordered=True)(phi[None], 2, dx + [1.0])[0])
    phi, src, dx = examples.extension_2d()
    dist = np.full_like(phi, np.nan)
    ext = [np.full_like(phi, np.nan) for _ in src]
    ext_p = (P * 2)(*[e.ctypes.data for e in ext])
    src_p = (P * 2)(*[s.ctypes.data for s in src])
    d, h = grid(phi, dx)
    assert e2(dist.ctypes.data, ctypes.cast(ext_p, P), phi.ctypes.data, None,
              ctypes.cast(src_p, P), None, 2, 2, d.ctypes.data, h.ctypes.data) == 0
    wd, wf = oracle.oracle_extension(ordered=True)(phi[None], [s[None] for s in src], 2, dx + [1.0])
    assert same_bits(dist, wd[0])
    for got, want in zip(ext, wf):
        assert same_bits(got, want[0])
    phi, speed, dx = examples.eikonal_2d()
    sol = phi.copy()
    d, h = grid(phi, dx)
    assert k2(sol.ctypes.data, speed.ctypes.data, None, 2, d.ctypes.data, h.ctypes.data) == 0
    assert same_bits(sol, oracle.oracle_eikonal(ordered=True)(phi[None], speed[None], 2, dx + [1.0])[0])
