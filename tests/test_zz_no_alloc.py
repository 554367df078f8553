"""The entry point that allocates nothing (lsmgpu_normal_rhs_dt_noalloc).

It serves callers that may not allocate device memory when they call in (a
fixed pre-reserved pool, a real-time loop, a framework that owns all device
memory).  Its scratch is a static device array, so these tests check, through
the C ABI, that two calls in a row give the same RHS and dt as the existing
reference-compatible entry points (LSM3D_HJ_WENO5 +
LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS and LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT):
bit for bit in strict mode, within 1e-12 relative in fast mode.  The second
call uses other inputs and a smaller fill box, so a stale value left in the
shared scratch by the first call would show."""
import ctypes

import numpy as np
import pytest

from lsmlib_b200.toolbox import Field

pytestmark = pytest.mark.gpu

PM = ("phi_x_plus", "phi_y_plus", "phi_z_plus", "phi_x_minus", "phi_y_minus",
      "phi_z_minus")


def make_case(n, lo, seed, speed_amp):
    rng = np.random.default_rng(seed)
    g = 3
    glo = tuple(l - g for l in lo)
    ghi = tuple(l + m - 1 + g for l, m in zip(lo, n))
    dx = (0.041, 0.037, 0.043)
    ax = [(np.arange(a, b + 1) + 0.5) * h for a, b, h in zip(glo, ghi, dx)]
    x, y, z = np.meshgrid(*ax, indexing="ij")
    phi = np.full(x.shape, np.inf)
    for _ in range(4):
        c = rng.uniform(0.2, 1.2, 3)
        phi = np.minimum(phi, np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 +
                                      (z - c[2]) ** 2) - rng.uniform(0.15, 0.35))
    F = 1.0 + speed_amp * np.sin(4 * np.pi * x) * np.sin(4 * np.pi * y) * np.sin(4 * np.pi * z)
    fb = (lo[0], lo[0] + n[0] - 1, lo[1], lo[1] + n[1] - 1, lo[2], lo[2] + n[2] - 1)
    return glo, ghi, fb, dx, np.asfortranarray(phi), np.asfortranarray(F)


def existing_path(tb, gpu, glo, ghi, fb, dx, phi, F):
    """RHS and dt through the reference-compatible entry points, on device."""
    d = {"phi": gpu.device_field(Field(phi, glo)),
         "vel_n": gpu.device_field(Field(F, glo)),
         "lse_rhs": gpu.device_field(Field.zeros(glo, ghi))}
    for nm in PM:
        d[nm] = gpu.device_field(Field.zeros(glo, ghi))
    sc = {"dx": dx[0], "dy": dx[1], "dz": dx[2]}
    for face in range(6):
        tb.call("lsm3dlinearextrapolation_", {"phi": d["phi"]}, fb,
                bdry_location_idx=face)
    tb.call("lsm3dzerooutlevelseteqnrhs_", {"lse_rhs": d["lse_rhs"]}, fb)
    tb.call("lsm3dhjweno5_", {k: d[k] for k in PM + ("phi",)}, fb, **sc)
    tb.call("lsm3daddnormalveltermtolserhs_",
            {k: d[k] for k in PM + ("lse_rhs", "vel_n")}, fb)
    dt = tb.call("lsm3dcomputestablenormalveldt_",
                 {k: d[k] for k in PM + ("vel_n",)}, fb, cfl_number=0.5, **sc)["dt"]
    return gpu.host_field(d["lse_rhs"]), dt, d["phi"]


def no_alloc_call(gpu, d_phi, d_F, glo, ghi, fb, dx, dt_on_device):
    from lsmlib_b200.ext_abi import dbls, ints
    lib = gpu.load()
    rhs = gpu.DeviceArray.from_host(np.zeros(tuple(h - l + 1 for l, h in zip(glo, ghi)),
                                             order="F"))
    gb = (glo[0], ghi[0], glo[1], ghi[1], glo[2], ghi[2])
    if dt_on_device:
        d_dt = gpu.DeviceArray((1, 1, 1))
        rc = lib.lsmgpu_normal_rhs_dt_noalloc(rhs.ptr, d_dt.ptr, d_phi.data.ptr,
                                              d_F.data.ptr, ints(gb), ints(fb),
                                              dbls(dx), 0.5)
        gpu.check_rc(rc, "noalloc")
        dt = float(d_dt.download().ravel()[0])
    else:
        h_dt = ctypes.c_double(-7.0)
        rc = lib.lsmgpu_normal_rhs_dt_noalloc(rhs.ptr, ctypes.byref(h_dt), d_phi.data.ptr,
                                              d_F.data.ptr, ints(gb), ints(fb),
                                              dbls(dx), 0.5)
        gpu.check_rc(rc, "noalloc")
        dt = h_dt.value
    return Field(rhs.download(), glo), dt


@pytest.mark.parametrize("mode", ["strict", "fast"])
def test_two_calls_match_existing_entry_points(gpu_tb, mode):
    from lsmlib_b200 import gpu, integrator
    prev = integrator.get_fp_mode()
    integrator.set_fp_mode(integrator.FP_STRICT if mode == "strict" else integrator.FP_FAST)
    try:
        cases = [((70, 45, 66), (-2, 1, 3), 5, 0.2, False),
                 ((33, 17, 21), (4, -6, 0), 9, 0.35, True)]
        for n, lo, seed, amp, dt_dev in cases:
            glo, ghi, fb, dx, phi, F = make_case(n, lo, seed, amp)
            want_rhs, want_dt, d_phi = existing_path(gpu_tb, gpu, glo, ghi, fb, dx, phi, F)
            d_F = gpu.device_field(Field(F, glo))
            got_rhs, got_dt = no_alloc_call(gpu, d_phi, d_F, glo, ghi, fb, dx, dt_dev)
            lo3, hi3 = (fb[0], fb[2], fb[4]), (fb[1], fb[3], fb[5])
            g, w = got_rhs.view(lo3, hi3), want_rhs.view(lo3, hi3)
            if mode == "strict":
                assert np.array_equal(g.view(np.uint64), w.view(np.uint64))
                assert got_dt == want_dt
            else:
                assert np.max(np.abs(g - w)) <= 1e-12 * np.max(np.abs(w))
                assert abs(got_dt - want_dt) <= 1e-12 * want_dt
    finally:
        integrator.set_fp_mode(prev)


def test_rejects_fill_box_beyond_the_static_scratch():
    from lsmlib_b200 import gpu
    from lsmlib_b200.ext_abi import dbls, ints
    lib = gpu.load()
    small = gpu.DeviceArray((4, 4, 4))
    fb = (0, 32 * 17 - 1, 0, 8 * 16 - 1, 0, 32 * 16 - 1)   # 17*16*32 = 8704 tiles > 8192
    gb = (-3, fb[1] + 3, -3, fb[3] + 3, -3, fb[5] + 3)
    dt = ctypes.c_double(0.0)
    rc = lib.lsmgpu_normal_rhs_dt_noalloc(small.ptr, ctypes.byref(dt), small.ptr,
                                          small.ptr, ints(gb), ints(fb),
                                          dbls((0.1, 0.1, 0.1)), 0.5)
    assert rc == 1
    msg = lib.lsmgpu_get_last_error_string().decode()
    assert "8192" in msg and "tiles" in msg
    lib.lsmgpu_get_last_error()


def test_rejects_tile_counts_that_wrap_32_bits():
    """2^17 x 2^15 x 1 tiles = 2^32: a 32-bit count would wrap to 0 and pass
    the size check.  The entry point counts in 64 bits and refuses the box
    before it looks at the arrays (host arrays here: nothing reaches the
    GPU)."""
    from lsmlib_b200 import gpu
    from lsmlib_b200.ext_abi import dbls, ints
    lib = gpu.load()
    a = np.zeros((4, 4, 4), order="F")
    fb = (0, 32 * 2 ** 17 - 1, 0, 8 * 2 ** 15 - 1, 0, 15)
    gb = (-3, fb[1] + 3, -3, fb[3] + 3, -3, fb[5] + 3)
    dt = ctypes.c_double(0.0)
    rc = lib.lsmgpu_normal_rhs_dt_noalloc(a.ctypes.data, ctypes.byref(dt), a.ctypes.data,
                                          a.ctypes.data, ints(gb), ints(fb),
                                          dbls((0.1, 0.1, 0.1)), 0.5)
    assert rc == 1
    msg = lib.lsmgpu_get_last_error_string().decode()
    assert "4294967296 tiles" in msg
    lib.lsmgpu_get_last_error()


def test_rejects_host_arrays():
    from lsmlib_b200 import gpu
    from lsmlib_b200.ext_abi import dbls, ints
    lib = gpu.load()
    a = np.zeros((12, 12, 12), order="F")
    dt = ctypes.c_double(0.0)
    rc = lib.lsmgpu_normal_rhs_dt_noalloc(a.ctypes.data, ctypes.byref(dt), a.ctypes.data,
                                          a.ctypes.data, ints((-3, 8, -3, 8, -3, 8)),
                                          ints((0, 5, 0, 5, 0, 5)),
                                          dbls((0.1, 0.1, 0.1)), 0.5)
    assert rc == 5
    lib.lsmgpu_get_last_error()
