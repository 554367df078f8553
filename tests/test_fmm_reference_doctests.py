"""The reference Python package's own known-answer doctests
(pylsmlib/pylsmlib/__init__.py:196-800) on the CPU checkers: the reference's
own fast marching routines (oracle/_ref/libfmm.so) and the oracle's heap
march (oracle/fmm_oracle.c), each driven through a restatement of the
reference package's wrapper (getShape, :25-57; lsmlib.pyx:10-120).  The GPU
runs the same cases through pylsmlib in tests/test_gpu_distance.py."""
import numpy as np
import pytest

import oracle
from fmm_reference_cases import CASES


class WrapperMirror:
    """computeDistanceFunction / computeExtensionFields / travel_time of the
    reference package over a C library's 3D entry points."""

    def __init__(self, dist, ext, eik):
        self.dist, self.ext, self.eik = dist, ext, eik

    @staticmethod
    def _grid(phi, dx):
        phi = np.asarray(phi, dtype=float)
        shape = phi.shape
        d = np.array(dx, dtype=float)
        if d.shape == ():
            d = np.resize(d, (len(shape),))
        if len(shape) == 1:
            nx, ny, hx, hy = shape[0], 1, d[0], 1.
        else:
            (ny, nx), (hy, hx) = shape, (d[0], d[1])
        return phi.reshape(1, ny, nx), (hx, hy, 1.), shape

    def distance(self, phi, dx, order):
        p3, h, shape = self._grid(phi, dx)
        return self.dist(p3, order, h).reshape(shape)

    def extension(self, phi, speed, dx, order, ext_mask):
        p3, h, shape = self._grid(phi, dx)
        u0 = np.asarray(speed, dtype=float)
        u0shape = u0.shape
        if u0shape == shape:
            u0 = u0.reshape((1,) + u0shape)
        em = None
        if ext_mask is not None:
            em = (-np.asarray(ext_mask, dtype=float) * 2. + 1.).reshape(p3.shape)
        dist, fields = self.ext(p3, [u.reshape(p3.shape) for u in u0], order, h, None, em)
        return dist.reshape(shape), np.stack(fields).reshape(u0shape)

    def travel_time(self, phi, speed, dx, order):
        p3, h, shape = self._grid(phi, dx)
        phi = p3.copy()
        minphi = phi.min()
        phi[phi > 0] = minphi - 1.
        phi = phi - minphi
        sol = self.eik(phi, np.asarray(speed, dtype=float).reshape(p3.shape), order, h)
        return abs((sol + minphi).reshape(shape))


def backends():
    out = [pytest.param("oracle", id="oracle"), pytest.param("ordered", id="ordered")]
    if oracle.fmm_available():
        out.insert(0, pytest.param("reference", id="reference"))
    return out


@pytest.fixture(scope="module", params=backends())
def backend(request):
    if request.param == "reference":
        return WrapperMirror(oracle.reference_fmm(), oracle.reference_extension(),
                             oracle.reference_eikonal())
    ordered = request.param == "ordered"   # the march the GPU solver computes
    return WrapperMirror(oracle.oracle_fmm(ordered), oracle.oracle_extension(ordered),
                         oracle.oracle_eikonal(ordered))


@pytest.mark.parametrize("case", CASES, ids=[c.__name__ for c in CASES])
def test_reference_doctest_case(backend, case):
    case(backend)
