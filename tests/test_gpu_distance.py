"""The GPU distance function (liblsmgpu.so computeDistanceFunction3d /
lsmgpu_distance_function3d) against the reference's fast marching method:
the committed golden outputs of the reference itself, and the C restatement
of its heap march (oracle/fmm_oracle.c) on seeded inputs, bit for bit."""
import ctypes

import numpy as np
import pytest

import oracle
from test_fmm_golden import GOLDEN, NAMES, _case, seeded_mask, seeded_spheres

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from lsmlib_b200 import gpu
    return gpu.load()


def gpu_distance(lib, phi, order, dx, mask=None):
    """lsmgpu_distance_function3d on host arrays (nz, ny, nx), dx in x, y, z."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    out = np.full_like(phi, np.nan)      # every cell is written: nothing is copied in
    dims = (ctypes.c_int * 3)(*phi.shape[::-1])
    h = (ctypes.c_double * 3)(*dx)
    passes = ctypes.c_int(0)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
    rc = lib.lsmgpu_distance_function3d(out.ctypes.data, phi.ctypes.data,
                                        None if m is None else m.ctypes.data, order, dims, h,
                                        ctypes.byref(passes))
    assert rc == 0, lib.lsmgpu_get_last_error_string()
    return out, passes.value


def same_bits(a, b):
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
def test_distance_reproduces_reference_golden(lib, name, order):
    z = np.load(GOLDEN)
    phi, dx, mask = _case(z, name)
    got, _ = gpu_distance(lib, phi, order, dx, mask)
    assert same_bits(got, z["%s|out%d" % (name, order)])


@pytest.mark.parametrize("shape,seed", [((33, 41, 29), 1), ((20, 64, 48), 2), ((1, 80, 90), 3),
                                        ((64, 64, 64), 4), ((40, 100, 70), 5)])
@pytest.mark.parametrize("order", [1, 2])
def test_distance_matches_oracle(lib, shape, seed, order):
    phi, dx = seeded_spheres(shape, seed)
    mask = seeded_mask(shape, seed)
    want = oracle.oracle_fmm(ordered=True)(phi, order, dx, mask)
    got, passes = gpu_distance(lib, phi, order, dx, mask)
    assert same_bits(got, want), (np.mean(got == want), np.abs(got - want).max())
    assert passes > 0


def test_distance_c_abi_entry_point(lib):
    """The reference's signature, host pointers, 0 on success and 2 for a bad
    order (lsm_fast_marching_method.h:386-392)."""
    z = np.load(GOLDEN)
    phi, dx, _ = _case(z, "spheres3d")
    fn = lib.computeDistanceFunction3d
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    phi = np.ascontiguousarray(phi)
    out = np.zeros_like(phi)
    dims = np.array(phi.shape[::-1], dtype=np.intc)
    h = np.array(dx)
    assert fn(out.ctypes.data, phi.ctypes.data, None, 2, dims.ctypes.data, h.ctypes.data) == 0
    assert same_bits(out, z["spheres3d|out2"])
    assert fn(out.ctypes.data, phi.ctypes.data, None, 3, dims.ctypes.data, h.ctypes.data) == 2


def test_distance_device_arrays(lib):
    """Device pointers are used in place (torch tensors on cuda:0)."""
    import torch
    phi, dx = seeded_spheres((24, 30, 36), 9)
    want = oracle.oracle_fmm(ordered=True)(phi, 2, dx)
    tp = torch.from_numpy(phi).cuda()
    out = torch.empty_like(tp)
    dims = (ctypes.c_int * 3)(*phi.shape[::-1])
    h = (ctypes.c_double * 3)(*dx)
    rc = lib.lsmgpu_distance_function3d(out.data_ptr(), tp.data_ptr(), None, 2, dims, h, None)
    assert rc == 0
    assert same_bits(out.cpu().numpy(), want)


def test_distance_after_scratch_release(lib):
    """The scratch the library keeps between calls can be handed back to the
    driver at any time; the next call maps new scratch and agrees bit for
    bit."""
    phi, dx = seeded_spheres((30, 26, 34), 10)
    first, _ = gpu_distance(lib, phi, 2, dx)
    assert lib.lsmgpu_release_scratch() == 0
    again, _ = gpu_distance(lib, phi, 2, dx)
    assert same_bits(first, again)
    assert same_bits(again, oracle.oracle_fmm(ordered=True)(phi, 2, dx))


def test_distance_edge_cases(lib):
    phi = np.ones((5, 6, 7))
    got, _ = gpu_distance(lib, phi, 1, [1.0, 1.0, 1.0])
    assert np.all(got == -1.0)                       # no interface: the default
    phi[2, 3, 3] = -1.0
    got, _ = gpu_distance(lib, phi, 2, [1.0, 1.0, 1.0], -np.ones_like(phi))
    assert np.all(got == np.finfo(np.float64).max)   # all outside the domain
    phi = np.linspace(-1, 1, 9)[None, None, :] * np.ones((3, 4, 9))
    got, _ = gpu_distance(lib, phi, 1, [0.25, 1.0, 1.0])
    assert same_bits(got, oracle.oracle_fmm(ordered=True)(phi, 1, [0.25, 1.0, 1.0]))
    assert np.all(got[..., 4] == -1e-11)             # on the interface
    one = np.array([[[0.3]]])                        # a single point
    got, _ = gpu_distance(lib, one, 2, [1.0, 1.0, 1.0])
    assert got[0, 0, 0] == -1.0


def test_pylsmlib_compute_distance_function():
    """The Python front door: C-ordered arrays, dx in shape order, 2D input."""
    from pylsmlib import computeDistanceFunction
    z = np.load(GOLDEN)
    phi = z["spheres2d|phi"][0]
    dx = z["spheres2d|dx"][1:]
    got = computeDistanceFunction(phi, dx, order=2)
    assert same_bits(got, z["spheres2d|out2"][0])
    got1 = computeDistanceFunction(phi[5], dx[1], order=1)      # 1D
    assert same_bits(got1, oracle.oracle_fmm(ordered=True)(phi[5][None, None, :], 1, [dx[1], 1.0, 1.0])[0, 0])


# ---- extension fields -------------------------------------------------------
from test_fmm_golden import ext_case, seeded_sources  # noqa: E402


def gpu_extension(lib, phi, sources, order, dx, mask=None, emask=None):
    """lsmgpu_extension_fields3d on host arrays: (distance, [fields])."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    src = [np.ascontiguousarray(a, dtype=np.float64) for a in sources]
    ext = [np.full_like(phi, np.nan) for _ in src]
    dist = np.full_like(phi, np.nan)
    nf = len(src)
    src_p = (ctypes.c_void_p * max(nf, 1))(*[a.ctypes.data for a in src])
    ext_p = (ctypes.c_void_p * max(nf, 1))(*[a.ctypes.data for a in ext])
    dims = (ctypes.c_int * 3)(*phi.shape[::-1])
    h = (ctypes.c_double * 3)(*dx)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
    em = None if emask is None else np.ascontiguousarray(emask, dtype=np.float64)
    rc = lib.lsmgpu_extension_fields3d(dist.ctypes.data, ctypes.cast(ext_p, ctypes.c_void_p),
                                       phi.ctypes.data, None if m is None else m.ctypes.data,
                                       ctypes.cast(src_p, ctypes.c_void_p),
                                       None if em is None else em.ctypes.data, nf, order, dims,
                                       h, None)
    assert rc == 0, lib.lsmgpu_get_last_error_string()
    return dist, ext


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
def test_extension_reproduces_reference_golden(lib, name, order):
    z = np.load(GOLDEN)
    phi, dx, mask = _case(z, name)
    src, emask = ext_case(z, name)
    dist, fields = gpu_extension(lib, phi, src, order, dx, mask, emask)
    assert same_bits(dist, z["%s|out%d" % (name, order)])
    for k, f in enumerate(fields):
        assert same_bits(f, z["%s|ext%d_%d" % (name, order, k)])


@pytest.mark.parametrize("shape,seed", [((33, 41, 29), 1), ((20, 64, 48), 2), ((1, 80, 90), 3),
                                        ((64, 64, 64), 4)])
@pytest.mark.parametrize("order", [1, 2])
def test_extension_matches_oracle(lib, shape, seed, order):
    phi, dx = seeded_spheres(shape, seed)
    mask = seeded_mask(shape, seed)
    emask = None
    if mask is not None:
        emask = np.where(np.random.default_rng(seed).random(shape) < 0.3, -1.0, 1.0)
    src = seeded_sources(shape, seed, n=3)
    want = oracle.oracle_extension(ordered=True)(phi, src, order, dx, mask, emask)
    got = gpu_extension(lib, phi, src, order, dx, mask, emask)
    assert same_bits(got[0], want[0])
    for a, b in zip(got[1], want[1]):
        assert same_bits(a, b), (np.mean(a == b), np.nanmax(np.abs(a - b)))


def test_extension_more_fields_than_one_solve(lib):
    """Nine fields: two groups of solves, each field as the oracle has it."""
    phi, dx = seeded_spheres((24, 28, 20), 6)
    src = seeded_sources((24, 28, 20), 6, n=9)
    want = oracle.oracle_extension(ordered=True)(phi, src, 2, dx)
    got = gpu_extension(lib, phi, src, 2, dx)
    assert same_bits(got[0], want[0])
    for a, b in zip(got[1], want[1]):
        assert same_bits(a, b)


def test_extension_c_abi_entry_point(lib):
    """computeExtensionFields3d with the reference's arguments (host arrays)
    and its return code 2 for a bad order."""
    z = np.load(GOLDEN)
    phi, dx, mask = _case(z, "masked3d")
    src, emask = ext_case(z, "masked3d")
    fn = lib.computeExtensionFields3d
    P = ctypes.c_void_p
    fn.restype = ctypes.c_int
    fn.argtypes = [P, P, P, P, P, P, ctypes.c_int, ctypes.c_int, P, P]
    phi = np.ascontiguousarray(phi)
    dist = np.full_like(phi, np.nan)
    ext = [np.full_like(phi, np.nan) for _ in src]
    src = [np.ascontiguousarray(a) for a in src]
    ext_p = (ctypes.c_void_p * 2)(*[a.ctypes.data for a in ext])
    src_p = (ctypes.c_void_p * 2)(*[a.ctypes.data for a in src])
    dims = np.array(phi.shape[::-1], dtype=np.intc)
    h = np.array(dx)
    m, em = np.ascontiguousarray(mask), np.ascontiguousarray(emask)
    args = [dist.ctypes.data, ctypes.cast(ext_p, P), phi.ctypes.data, m.ctypes.data,
            ctypes.cast(src_p, P), em.ctypes.data, 2]
    assert fn(*args, 1, dims.ctypes.data, h.ctypes.data) == 0
    assert same_bits(dist, z["masked3d|out1"])
    assert same_bits(ext[0], z["masked3d|ext1_0"]) and same_bits(ext[1], z["masked3d|ext1_1"])
    assert fn(*args, 3, dims.ctypes.data, h.ctypes.data) == 2


def test_pylsmlib_compute_extension_fields():
    """The Python front door: (N,) + shape speeds, boolean ext_mask."""
    from pylsmlib import computeExtensionFields
    phi, dx = seeded_spheres((1, 40, 50), 8)
    phi2 = phi[0]
    src = seeded_sources((1, 40, 50), 8, n=2)
    speed = np.stack([a[0] for a in src])
    em = np.random.default_rng(3).random(phi2.shape) < 0.2
    dist, ext = computeExtensionFields(phi2, speed, dx=[dx[1], dx[0]], order=1, ext_mask=em)
    want = oracle.oracle_extension(ordered=True)(phi, src, 1, dx, None,
                                     (-em.astype(float) * 2.0 + 1.0)[None])
    assert same_bits(dist, want[0][0])
    assert ext.shape == speed.shape
    for k in range(2):
        assert same_bits(ext[k], want[1][k][0])


# ---- Eikonal solver -------------------------------------------------------------
from test_fmm_golden import eik_case, seeded_eikonal  # noqa: E402


def gpu_eikonal(lib, data, speed, order, dx, mask=None):
    """lsmgpu_eikonal3d on host arrays: the solution (a new array)."""
    phi = np.array(data, dtype=np.float64, order="C", copy=True)
    f = np.ascontiguousarray(speed, dtype=np.float64)
    dims = (ctypes.c_int * 3)(*phi.shape[::-1])
    h = (ctypes.c_double * 3)(*dx)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
    rc = lib.lsmgpu_eikonal3d(phi.ctypes.data, f.ctypes.data,
                              None if m is None else m.ctypes.data, order, dims, h, None)
    assert rc == 0, lib.lsmgpu_get_last_error_string()
    return phi


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("order", [1, 2])
def test_eikonal_reproduces_reference_golden(lib, name, order):
    z = np.load(GOLDEN)
    data, speed, mask = eik_case(z, name)
    got = gpu_eikonal(lib, data, speed, order, z[name + "|dx"][::-1], mask)
    assert same_bits(got, z["%s|eik%d" % (name, order)])


@pytest.mark.parametrize("shape,seed", [((33, 41, 29), 1), ((20, 64, 48), 2), ((1, 80, 90), 3),
                                        ((64, 64, 64), 4), ((40, 100, 70), 5)])
@pytest.mark.parametrize("order", [1, 2])
def test_eikonal_matches_oracle(lib, shape, seed, order):
    data, speed, dx = seeded_eikonal(shape, seed)
    mask = seeded_mask(shape, seed)
    want = oracle.oracle_eikonal(ordered=True)(data, speed, order, dx, mask)
    got = gpu_eikonal(lib, data, speed, order, dx, mask)
    assert same_bits(got, want), (np.mean(got == want), np.abs(got - want).max())


def test_eikonal_c_abi_entry_point(lib):
    """solveEikonalEquation3d with the reference's arguments: phi in/out on
    the device, 2 for a bad order."""
    import torch
    data, speed, dx = seeded_eikonal((24, 30, 36), 9)
    want = oracle.oracle_eikonal(ordered=True)(data, speed, 2, dx)
    fn = lib.solveEikonalEquation3d
    P = ctypes.c_void_p
    fn.restype = ctypes.c_int
    fn.argtypes = [P, P, P, ctypes.c_int, P, P]
    tp = torch.from_numpy(np.ascontiguousarray(data)).cuda()
    tf = torch.from_numpy(np.ascontiguousarray(speed)).cuda()
    dims = np.array(data.shape[::-1], dtype=np.intc)
    h = np.array(dx)
    assert fn(tp.data_ptr(), tf.data_ptr(), None, 2, dims.ctypes.data, h.ctypes.data) == 0
    assert same_bits(tp.cpu().numpy(), want)
    assert fn(tp.data_ptr(), tf.data_ptr(), None, 0, dims.ctypes.data, h.ctypes.data) == 2


def test_pylsmlib_solve_eikonal_equation():
    """The Python front door shifts phi as the reference's wrapper does."""
    from pylsmlib import solveEikonalEquation, travel_time
    sdf, dx = seeded_spheres((1, 40, 50), 12, noise=0.0)
    speed = 1.0 + 0.25 * np.cos(np.linspace(0, 7, sdf.size)).reshape(sdf.shape)
    minphi = sdf.min()
    data = np.where(sdf > 0, minphi - 1.0, sdf) - minphi
    want = oracle.oracle_eikonal(ordered=True)(data, speed, 2, dx) + minphi
    got = solveEikonalEquation(sdf[0], speed[0], dx=[dx[1], dx[0]], order=2)
    assert same_bits(got, want[0])
    assert same_bits(travel_time(sdf[0], speed[0], dx=[dx[1], dx[0]]), np.abs(want[0]))

