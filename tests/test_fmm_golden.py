"""The checkers for the distance function.

* The reference's own fast marching method, built from its C sources
  (oracle/_ref/libfmm.so), reproduces the committed golden outputs bit for
  bit (these pin the fixtures to the reference).
* The C restatement of the heap march (oracle/fmm_oracle.c) reproduces the
  same golden outputs, and the reference's results on seeded noisy unions of
  spheres, bit for bit (these pin the restatement).
* The same for the extension fields (computeExtensionFields3d) and the
  Eikonal solver (solveEikonalEquation3d).
* The ordered march (the same march popping exact key ties by acceptance
  time and then point index, which the GPU solver computes) equals the
  reference on every case without exact ties: the golden and seeded cases
  above are run through it too.  Where keys tie (the reference's own
  symmetric examples), the two differ only by the order in which tied
  points are accepted (test_tied_keys_*).
"""
import ctypes
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fmm_golden.npz")
NAMES = ("spheres3d", "masked3d", "spheres2d")


def _case(z, name):
    """phi (nz, ny, nx), dx in x, y, z order, mask or None."""
    mask = z[name + "|mask"] if name + "|mask" in z.files else None
    return z[name + "|phi"], z[name + "|dx"][::-1], mask


def seeded_spheres(shape, seed, noise=0.01):
    """A noisy union of two spheres on [-1, 1] per axis: phi (nz, ny, nx) and
    dx in x, y, z order (an axis of one point gets dx 1)."""
    rng = np.random.default_rng(seed)
    axes = [np.linspace(-1, 1, n) if n > 1 else np.zeros(1) for n in shape]
    zz, yy, xx = np.meshgrid(*axes, indexing="ij")
    c = rng.uniform(-0.3, 0.3, size=(2, 3))
    r = rng.uniform(0.25, 0.5, size=2)
    phi = np.minimum(np.sqrt((xx - c[0, 0]) ** 2 + (yy - c[0, 1]) ** 2 + (zz - c[0, 2]) ** 2) - r[0],
                     np.sqrt((xx - c[1, 0]) ** 2 + (yy - c[1, 1]) ** 2 + (zz - c[1, 2]) ** 2) - r[1])
    if noise:
        phi = phi + noise * rng.standard_normal(shape)
    dx = [2.0 / (n - 1) if n > 1 else 1.0 for n in shape[::-1]]
    return phi, dx


def seeded_mask(shape, seed):
    """Outside-domain block for the masked seeded cases (None otherwise)."""
    if seed != 2:
        return None
    mask = np.ones(shape)
    mask[:, 5:20, 3:11] = -1.0
    return mask


@pytest.mark.skipif(not oracle.fmm_available(), reason="oracle/_ref/libfmm.so not built")
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
def test_reference_fmm_reproduces_golden(name, order):
    z = np.load(GOLDEN)
    phi, dx, mask = _case(z, name)
    got = oracle.reference_fmm()(phi, order, dx, mask)
    assert np.array_equal(got.view(np.uint64), z["%s|out%d" % (name, order)].view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("ordered", [False, True], ids=["heap", "ordered"])
def test_oracle_fmm_reproduces_golden(name, order, ordered):
    z = np.load(GOLDEN)
    phi, dx, mask = _case(z, name)
    got = oracle.oracle_fmm(ordered)(phi, order, dx, mask)
    assert np.array_equal(got.view(np.uint64), z["%s|out%d" % (name, order)].view(np.uint64))


@pytest.mark.skipif(not oracle.fmm_available(), reason="oracle/_ref/libfmm.so not built")
@pytest.mark.parametrize("shape,seed", [((33, 41, 29), 1), ((20, 64, 48), 2), ((1, 80, 90), 3)])
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("ordered", [False, True], ids=["heap", "ordered"])
def test_oracle_fmm_matches_reference(shape, seed, order, ordered):
    phi, dx = seeded_spheres(shape, seed)
    mask = seeded_mask(shape, seed)
    a = oracle.oracle_fmm(ordered)(phi, order, dx, mask)
    b = oracle.reference_fmm()(phi, order, dx, mask)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_oracle_fmm_edge_cases():
    fmm = oracle.oracle_fmm()
    # no interface: no front, every point keeps the default -1
    phi = np.ones((5, 6, 7))
    assert np.all(fmm(phi, 1, [1.0, 1.0, 1.0]) == -1.0)
    # a mask that excludes everything: LSMLIB_REAL_MAX everywhere
    phi[2, 3, 3] = -1.0
    out = fmm(phi, 2, [1.0, 1.0, 1.0], -np.ones_like(phi))
    assert np.all(out == np.finfo(np.float64).max)
    # points exactly on the interface hold -1e-11 (LSMLIB_ZERO_TOL, phi = 0
    # is not > 0); the next ones are one and two cells away
    phi = np.linspace(-1, 1, 9)[None, None, :] * np.ones((3, 4, 9))
    out = fmm(phi, 1, [0.25, 1.0, 1.0])
    assert np.all(out[..., 4] == -1e-11)
    assert np.all(out[..., 5] == 0.25) and np.all(out[..., 6] == 0.5)
    # an order other than 1 or 2 is refused with the reference's code 2
    with pytest.raises(RuntimeError, match="returned 2"):
        fmm(phi, 3, [1.0, 1.0, 1.0])


def ext_case(z, name):
    """Source fields and extension mask (or None) of a golden case."""
    src = [z["%s|src%d" % (name, k)] for k in range(2)]
    emask = z[name + "|emask"] if name + "|emask" in z.files else None
    return src, emask


def seeded_sources(shape, seed, n=2):
    rng = np.random.default_rng(seed + 100)
    out = [rng.standard_normal(shape)]
    x = np.arange(np.prod(shape), dtype=np.float64).reshape(shape)
    out += [np.cos(0.01 * (k + 1) * x) for k in range(n - 1)]
    return out


@pytest.mark.skipif(not oracle.fmm_available(), reason="oracle/_ref/libfmm.so not built")
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
def test_reference_extension_reproduces_golden(name, order):
    z = np.load(GOLDEN)
    phi, dx, mask = _case(z, name)
    src, emask = ext_case(z, name)
    dist, fields = oracle.reference_extension()(phi, src, order, dx, mask, emask)
    assert np.array_equal(dist.view(np.uint64), z["%s|out%d" % (name, order)].view(np.uint64))
    for k, f in enumerate(fields):
        assert np.array_equal(f.view(np.uint64), z["%s|ext%d_%d" % (name, order, k)].view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("ordered", [False, True], ids=["heap", "ordered"])
def test_oracle_extension_reproduces_golden(name, order, ordered):
    z = np.load(GOLDEN)
    phi, dx, mask = _case(z, name)
    src, emask = ext_case(z, name)
    dist, fields = oracle.oracle_extension(ordered)(phi, src, order, dx, mask, emask)
    assert np.array_equal(dist.view(np.uint64), z["%s|out%d" % (name, order)].view(np.uint64))
    for k, f in enumerate(fields):
        assert np.array_equal(f.view(np.uint64), z["%s|ext%d_%d" % (name, order, k)].view(np.uint64))


@pytest.mark.skipif(not oracle.fmm_available(), reason="oracle/_ref/libfmm.so not built")
@pytest.mark.parametrize("shape,seed", [((33, 41, 29), 1), ((20, 64, 48), 2), ((1, 50, 60), 3)])
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("ordered", [False, True], ids=["heap", "ordered"])
def test_oracle_extension_matches_reference(shape, seed, order, ordered):
    phi, dx = seeded_spheres(shape, seed)
    mask = seeded_mask(shape, seed)
    emask = None
    if mask is not None:
        emask = np.where(np.random.default_rng(seed).random(shape) < 0.3, -1.0, 1.0)
    src = seeded_sources(shape, seed)
    a = oracle.reference_extension()(phi, src, order, dx, mask, emask)
    b = oracle.oracle_extension(ordered)(phi, src, order, dx, mask, emask)
    for x, y in zip([a[0]] + a[1], [b[0]] + b[1]):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))


def eik_case(z, name):
    """Boundary data, speed and mask of a golden Eikonal case."""
    from gen_fmm_golden import eikonal_case
    phi, _, mask = _case(z, name)
    data, speed = eikonal_case(name, phi, mask)
    return data, speed, mask


def seeded_eikonal(shape, seed):
    """Boundary data (phi <= 0 of seeded spheres, shifted as the reference's
    Python wrapper does), a speed with a zero-speed slab, dx."""
    sdf, dx = seeded_spheres(shape, seed, noise=0.0)
    minphi = sdf.min()
    data = np.where(sdf > 0, minphi - 1.0, sdf) - minphi
    x = np.linspace(0.0, 1.0, sdf.size).reshape(shape)
    speed = 1.0 + 0.5 * np.sin(40 * x)
    if shape[1] > 44:
        speed[:, 40:44, :] = 0.0
    return data, speed, dx


@pytest.mark.skipif(not oracle.fmm_available(), reason="oracle/_ref/libfmm.so not built")
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
def test_reference_eikonal_reproduces_golden(name, order):
    z = np.load(GOLDEN)
    data, speed, mask = eik_case(z, name)
    got = oracle.reference_eikonal()(data, speed, order, z[name + "|dx"][::-1], mask)
    assert np.array_equal(got.view(np.uint64), z["%s|eik%d" % (name, order)].view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("ordered", [False, True], ids=["heap", "ordered"])
def test_oracle_eikonal_reproduces_golden(name, order, ordered):
    z = np.load(GOLDEN)
    data, speed, mask = eik_case(z, name)
    got = oracle.oracle_eikonal(ordered)(data, speed, order, z[name + "|dx"][::-1], mask)
    assert np.array_equal(got.view(np.uint64), z["%s|eik%d" % (name, order)].view(np.uint64))


@pytest.mark.skipif(not oracle.fmm_available(), reason="oracle/_ref/libfmm.so not built")
@pytest.mark.parametrize("shape,seed", [((33, 41, 29), 1), ((20, 64, 48), 2), ((1, 50, 60), 3)])
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("ordered", [False, True], ids=["heap", "ordered"])
def test_oracle_eikonal_matches_reference(shape, seed, order, ordered):
    data, speed, dx = seeded_eikonal(shape, seed)
    mask = seeded_mask(shape, seed)
    a = oracle.reference_eikonal()(data, speed, order, dx, mask)
    b = oracle.oracle_eikonal(ordered)(data, speed, order, dx, mask)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
def test_golden_distance_sign_follows_phi(name, order):
    z = np.load(GOLDEN)
    phi, d = z[name + "|phi"], z["%s|out%d" % (name, order)]
    inside = np.abs(d) < 1e300
    sel = inside & (np.abs(phi) > 1e-9)
    assert np.all(np.sign(d[sel]) == np.sign(phi[sel]))


def test_pylsmlib_distance_argument_errors():
    """The reference pylsmlib's ValueErrors, raised before any GPU work."""
    from pylsmlib import computeDistanceFunction
    phi = np.zeros((4, 5))
    with pytest.raises(ValueError, match="dx must be of length"):
        computeDistanceFunction(phi, dx=[1.0, 1.0, 1.0])
    with pytest.raises(ValueError, match="greater than zero"):
        computeDistanceFunction(phi, dx=[1.0, 0.0])
    with pytest.raises(ValueError, match="order must be 1 or 2"):
        computeDistanceFunction(phi, dx=1.0, order=3)
    with pytest.raises(ValueError, match="mask"):
        computeDistanceFunction(phi, dx=1.0, mask=np.ones((5, 4)))


def test_pylsmlib_reference_doctest_errors():
    """The argument errors of the reference package's own doctests
    (pylsmlib/pylsmlib/__init__.py:442-449, 504-511, 625-635, 770-794), with
    their messages; all are raised before any GPU work."""
    from pylsmlib import computeDistanceFunction as distance
    from pylsmlib import computeExtensionFields, travel_time
    with pytest.raises(ValueError, match="dx must be of length len"):
        distance([[-1, 1], [1, 1]], dx=(1, 2, 3))
    with pytest.raises(ValueError, match="phi and speed must have the same shape"):
        computeExtensionFields([[-1, 1], [1, 1]], speed=[1, 1])
    for order in (0, 3):
        with pytest.raises(ValueError, match="order must be 1 or 2"):
            distance([-1, 1], order=order)
    with pytest.raises(ValueError, match="dx must be greater than zero"):
        distance([1, 0, 1, 1], 0)
    with pytest.raises(ValueError, match="dx must be of length len"):
        distance([0, 0, 1, 0, 0], [0, 0, 1, 0, 0])
    with pytest.raises(ValueError, match="phi and speed must have the same shape"):
        travel_time([-1, 1], [2])
    with pytest.raises(ValueError, match="phi and speed must have the same shape"):
        travel_time([0, 0, 1, 1], 2)
    with pytest.raises(ValueError, match="dx must be of length len"):
        travel_time([-1, 1], [2, 2], [2, 2, 2, 2])
    with pytest.raises(ValueError, match="could not convert string to float"):
        distance(np.array(["a", "b"]))


def _ref_2d_and_3d():
    lib = ctypes.CDLL(oracle.FMM_SO)
    if not hasattr(lib, "computeDistanceFunction2d"):
        pytest.skip("oracle/_ref/libfmm.so built without the 2D sources")
    return lib


@pytest.mark.parametrize("shape,seed,noise", [((30, 40), 3, 0.0), ((57, 41), 5, 0.01),
                                              ((33, 64), 9, 0.01)])
@pytest.mark.parametrize("order", [1, 2])
def test_reference_2d_routines_equal_3d_on_one_plane(shape, seed, order, noise):
    """The reference's 2D routines (lsm_fast_marching_method.h:124-262) give
    bit for bit what its 3D routines give on a grid one plane thick. So the
    2D entry points of the GPU library, which run the 3D solve on such a
    grid, inherit the 3D parity."""
    lib = _ref_2d_and_3d()
    P = ctypes.c_void_p
    ny, nx = shape
    phi3, dx = seeded_spheres((1, ny, nx), seed, noise=noise)
    phi = np.ascontiguousarray(phi3[0])
    d2, d3 = np.array([nx, ny], dtype=np.intc), np.array([nx, ny, 1], dtype=np.intc)
    h2, h3 = np.array(dx[:2]), np.array(dx)
    a, b = np.zeros_like(phi), np.zeros_like(phi)
    assert lib.computeDistanceFunction2d(a.ctypes.data_as(P), phi.ctypes.data_as(P), None, order,
                                         d2.ctypes.data_as(P), h2.ctypes.data_as(P)) == 0
    assert lib.computeDistanceFunction3d(b.ctypes.data_as(P), phi.ctypes.data_as(P), None, order,
                                         d3.ctypes.data_as(P), h3.ctypes.data_as(P)) == 0
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    # extension fields: two sources
    src = [np.ascontiguousarray(np.sin(3 * np.arange(phi.size)).reshape(phi.shape)),
           np.ascontiguousarray(np.cos(np.arange(phi.size) / 7.0).reshape(phi.shape))]
    outs = []
    for d, h, fn in ((d2, h2, lib.computeExtensionFields2d), (d3, h3, lib.computeExtensionFields3d)):
        dist = np.zeros_like(phi)
        ext = [np.zeros_like(phi) for _ in src]
        ext_p = (P * 2)(*[e.ctypes.data for e in ext])
        src_p = (P * 2)(*[s_.ctypes.data for s_ in src])
        assert fn(dist.ctypes.data_as(P), ext_p, phi.ctypes.data_as(P), None, src_p, None, 2,
                  order, d.ctypes.data_as(P), h.ctypes.data_as(P)) == 0
        outs.append([dist] + ext)
    for x, y in zip(*outs):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
    # Eikonal: phi <= 0 (shifted) as boundary data, varying speed
    m = phi.min()
    yy, xx = np.meshgrid(np.linspace(-1, 1, ny), np.linspace(-1, 1, nx), indexing="ij")
    speed = np.ascontiguousarray(1 + 0.5 * np.sin(3 * xx) * np.cos(2 * yy))
    e2 = np.ascontiguousarray(np.where(phi > 0, m - 1.0, phi) - m)
    e3 = e2.copy()
    assert lib.solveEikonalEquation2d(e2.ctypes.data_as(P), speed.ctypes.data_as(P), None, order,
                                      d2.ctypes.data_as(P), h2.ctypes.data_as(P)) == 0
    assert lib.solveEikonalEquation3d(e3.ctypes.data_as(P), speed.ctypes.data_as(P), None, order,
                                      d3.ctypes.data_as(P), h3.ctypes.data_as(P)) == 0
    assert np.array_equal(e2.view(np.uint64), e3.view(np.uint64))


# ---- the reference's fast marching examples ------------------------------------

import fmm_example_cases as examples  # noqa: E402


def _plane(a):
    return np.ascontiguousarray(a)[None]


@pytest.mark.skipif(not oracle.fmm_available(), reason="oracle/_ref/libfmm.so not built")
def test_reference_examples_oracle_matches_reference():
    """The inputs of examples/serial/fast_marching_method/*.c through the
    routines each example calls (the 2D ones for the 2D examples), against
    the oracle's 3D march (one plane thick for 2D), bit for bit."""
    lib = _ref_2d_and_3d()
    P = ctypes.c_void_p
    phi, dx = examples.distance_3d()
    want = oracle.oracle_fmm()(phi, 2, dx)
    assert np.array_equal(oracle.reference_fmm()(phi, 2, dx).view(np.uint64),
                          want.view(np.uint64))
    phi, dx = examples.distance_2d()
    out = np.zeros_like(phi)
    d = np.array(phi.shape[::-1], dtype=np.intc)
    h = np.array(dx)
    assert lib.computeDistanceFunction2d(out.ctypes.data_as(P), phi.ctypes.data_as(P), None, 2,
                                         d.ctypes.data_as(P), h.ctypes.data_as(P)) == 0
    want = oracle.oracle_fmm()(_plane(phi), 2, dx + [1.0])[0]
    assert np.array_equal(out.view(np.uint64), want.view(np.uint64))
    phi, src, dx = examples.extension_2d()
    dist = np.zeros_like(phi)
    ext = [np.zeros_like(phi) for _ in src]
    ext_p = (P * 2)(*[e.ctypes.data for e in ext])
    src_p = (P * 2)(*[s_.ctypes.data for s_ in src])
    d = np.array(phi.shape[::-1], dtype=np.intc)
    h = np.array(dx)
    assert lib.computeExtensionFields2d(dist.ctypes.data_as(P), ext_p, phi.ctypes.data_as(P),
                                        None, src_p, None, 2, 2, d.ctypes.data_as(P),
                                        h.ctypes.data_as(P)) == 0
    wd, wf = oracle.oracle_extension()(_plane(phi), [_plane(s_) for s_ in src], 2, dx + [1.0])
    for got, want in zip([dist] + ext, [wd[0]] + [f[0] for f in wf]):
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    phi, speed, dx = examples.eikonal_2d()
    sol = phi.copy()
    d = np.array(phi.shape[::-1], dtype=np.intc)
    h = np.array(dx)
    assert lib.solveEikonalEquation2d(sol.ctypes.data_as(P), speed.ctypes.data_as(P), None, 2,
                                      d.ctypes.data_as(P), h.ctypes.data_as(P)) == 0
    want = oracle.oracle_eikonal()(_plane(phi), _plane(speed), 2, dx + [1.0])[0]
    assert np.array_equal(sol.view(np.uint64), want.view(np.uint64))


# ---- exact key ties: the reference's heap order against the ordered march ------

def _quantised(shape, seed):
    phi, dx = seeded_spheres(shape, seed)
    return np.round(phi * 8) / 8, dx


@pytest.mark.parametrize("order", [1, 2])
def test_tied_keys_distance_examples_unaffected(order):
    """The reference's distance and extension examples hold ties that do not
    change any value: the ordered march gives the heap march's result bit for
    bit on them."""
    for phi, dx in (examples.distance_3d(), examples.distance_2d()):
        phi = phi if phi.ndim == 3 else _plane(phi)
        dx = list(dx) + [1.0] * (3 - len(dx))
        a = oracle.oracle_fmm()(phi, order, dx)
        b = oracle.oracle_fmm(True)(phi, order, dx)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    phi, src, dx = examples.extension_2d()
    a = oracle.oracle_extension()(_plane(phi), [_plane(s_) for s_ in src], order, dx + [1.0])
    b = oracle.oracle_extension(True)(_plane(phi), [_plane(s_) for s_ in src], order, dx + [1.0])
    for x, y in zip([a[0]] + a[1], [b[0]] + b[1]):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))


def test_tied_keys_first_order_differ_by_rounding_only():
    """At first order a tie only decides whether a neighbour of equal value
    joins an update, which leaves the root unchanged up to rounding: the
    heap's order and the ordered march agree to 1e-13 relative (the
    reference's 2D Eikonal example, quantised distance data)."""
    phi, speed, dx = examples.eikonal_2d()
    a = oracle.oracle_eikonal()(_plane(phi), _plane(speed), 1, dx + [1.0])
    b = oracle.oracle_eikonal(True)(_plane(phi), _plane(speed), 1, dx + [1.0])
    assert not np.array_equal(a, b)
    assert np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-300)) < 1e-13
    for seed in (1, 3):
        phi, dx = _quantised((17, 23, 19), seed)
        a = oracle.oracle_fmm()(phi, 1, dx)
        b = oracle.oracle_fmm(True)(phi, 1, dx)
        assert np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-300)) < 1e-13


def test_tied_keys_second_order_stencil_choice():
    """At second order a tie can decide whether the next point along an axis
    was KNOWN at an update, i.e. whether that axis takes the second-order
    stencil, so the two orders of acceptance give two different valid
    solutions.  On the reference's 2D Eikonal example (solveEikonalEquation2d.c:
    a disk of zeros, speed 1 / 2 split at x = 0, mirror-symmetric in y) the
    first difference is at a point whose +y neighbours at distance 1 and 2
    carry the same key; both results stay within 1e-2 of each other."""
    phi, speed, dx = examples.eikonal_2d()
    a = oracle.oracle_eikonal()(_plane(phi), _plane(speed), 2, dx + [1.0])[0]
    b = oracle.oracle_eikonal(True)(_plane(phi), _plane(speed), 2, dx + [1.0])[0]
    assert not np.array_equal(a, b)
    assert np.max(np.abs(a - b)) < 1e-2
    # (x, y) = (75, 43): keys of (75, 44) and (75, 45) are both 1/150
    assert a[44, 75] == b[44, 75] == a[45, 75] == b[45, 75]
    assert a[43, 75] != b[43, 75]
