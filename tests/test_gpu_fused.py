"""Fused TVD-RK3 stages and drivers against the oracle's reference-order chain.

Strict mode (reference expression order, no FMA) must be bit-identical to the
chain ghost fill -> zero RHS -> WENO5 -> RHS term -> TVD-RK3 stage of the
oracle; fast mode must stay within 1e-12 of it (relative max-norm:
max|gpu - ref| / max|ref|); the FP32 form within 1e-5 of the FP64 oracle."""
import numpy as np
import pytest

import oracle
from oracle.driver import Grid, Stepper, deformation_velocity

pytestmark = pytest.mark.gpu

REL_FAST = 1e-12
ABS_FP32 = 1e-5


def rel_err(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


def sphere(g, x_lo, c=(0.1, -0.05, 0.0), r=0.25):
    x, y, z = g.centers(x_lo)
    return np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - r


def spheres(g, x_lo, seed, count=6):
    rng = np.random.default_rng(seed)
    x, y, z = g.centers(x_lo)
    phi = np.full(g.shape, np.inf)
    for _ in range(count):
        c = rng.uniform(-0.6, 0.6, 3)
        r = rng.uniform(0.1, 0.3)
        phi = np.minimum(phi, np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - r)
    return phi


def same_bits(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64),
                          np.ascontiguousarray(b).view(np.uint64))


@pytest.fixture(params=["strict", "fast"])
def mode(request):
    from lsmlib_b200 import integrator
    prev = integrator.get_fp_mode()
    integrator.set_fp_mode(integrator.FP_STRICT if request.param == "strict"
                           else integrator.FP_FAST)
    yield request.param
    integrator.set_fp_mode(prev)


def check(mode, got, want):
    if mode == "strict":
        assert same_bits(got, want), "max diff %g" % np.max(np.abs(got - want))
    else:
        assert rel_err(got, want) <= REL_FAST


GRIDS = [(37, 11, 35), (16, 16, 16), (64, 9, 33)]


@pytest.mark.parametrize("n", GRIDS)
def test_advect_constant_velocity(mode, n):
    from lsmlib_b200 import gpu, integrator
    g = Grid(n, dx=(2.0 / n[0], 2.0 / n[1], 2.0 / n[2]))
    x_lo = (-1.0, -1.0, -1.0)
    phi0 = sphere(g, x_lo)
    vel = [g.field(np.full(g.shape, c)) for c in (1.0, 0.5, -0.25)]
    st = Stepper(oracle.oracle_toolbox(), g)
    ref = g.field(phi0)
    dt = st.advect_dt(vel, 0.5)
    for _ in range(3):
        st.advect_step(ref, lambda c: vel, dt)
    ws = integrator.Workspace(g.gb, 8)
    d = gpu.DeviceArray.from_host(phi0)
    dv = [gpu.DeviceArray.from_host(v.data) for v in vel]
    ws.advect(d, dv, g.fb, g.dx, cfl=0.5, nsteps=3)
    t, dt_last = ws.time()
    assert dt_last == dt
    check(mode, g.interior(g.field(d.download())), g.interior(ref))


@pytest.mark.parametrize("n", [(24, 20, 18), (33, 17, 40)])
def test_advect_random_velocity_field(mode, n):
    """Velocity with sign changes and exact zeros exercises every upwind
    branch (zero, backward, forward)."""
    from lsmlib_b200 import gpu, integrator
    rng = np.random.default_rng(7)
    g = Grid(n, dx=(0.05, 0.06, 0.07))
    phi0 = spheres(g, (-0.6, -0.6, -0.6), seed=3)
    vel = []
    for _ in range(3):
        v = rng.standard_normal(g.shape)
        v[rng.random(g.shape) < 0.1] = 0.0
        vel.append(g.field(v))
    st = Stepper(oracle.oracle_toolbox(), g)
    ref = g.field(phi0)
    dt = 0.01
    for _ in range(2):
        st.advect_step(ref, lambda c: vel, dt)
    ws = integrator.Workspace(g.gb, 8)
    d = gpu.DeviceArray.from_host(phi0)
    dv = [gpu.DeviceArray.from_host(v.data) for v in vel]
    ws.advect(d, dv, g.fb, g.dx, dt_fixed=dt, nsteps=2)
    check(mode, g.interior(g.field(d.download())), g.interior(ref))


@pytest.mark.parametrize("n", [(32, 24, 20), (19, 33, 17)])
def test_normal_velocity_with_reinitialization(mode, n):
    from lsmlib_b200 import gpu, integrator
    g = Grid(n, dx=(2.0 / n[0],) * 3)
    x_lo = (-1.0, -1.0, -1.0)
    phi0 = spheres(g, x_lo, seed=11)
    x, y, z = g.centers(x_lo)
    F = 1.0 + 0.2 * np.sin(4 * np.pi * x) * np.sin(4 * np.pi * y) * np.sin(4 * np.pi * z)
    Ff = g.field(F)
    st = Stepper(oracle.oracle_toolbox(), g)
    ref = g.field(phi0)
    for s in range(4):
        st.normal_step(ref, Ff, 0.5)
        if (s + 1) % 2 == 0:
            st.reinit(ref, 0.5, 3, use0=0)
    ws = integrator.Workspace(g.gb, 8)
    d = gpu.DeviceArray.from_host(phi0)
    dF = gpu.DeviceArray.from_host(F)
    ws.normal(d, dF, g.fb, g.dx, cfl=0.5, nsteps=4, reinit_interval=2,
              reinit_iters=3, use_phi0=0)
    check(mode, g.interior(g.field(d.download())), g.interior(ref))


def test_config2_fast_mode_at_128_cubed():
    """The benchmark's workload (6 seeded spheres, F = 1 + 0.2 sin sin sin,
    CFL 0.5) at 128^3 in the benchmark's arithmetic (fast mode): 3 steps, then
    2 reinitialization pseudo-steps, against the oracle's chain of the
    reference's routines in the reference integrators' order
    (LevelSetFunctionIntegrator.cc:1319-1510, ReinitializationAlgorithm.cc:
    177-330), run over z-slab patches on the host cores."""
    import os

    from lsmlib_b200 import gpu, integrator, workloads
    from oracle.driver import PatchedNormalStepper
    cfg = workloads.config2(128)
    gb, fb = workloads.boxes(cfg["n"])
    prev = integrator.get_fp_mode()
    integrator.set_fp_mode(integrator.FP_FAST)
    try:
        ws = integrator.Workspace(gb, 8)
        d = gpu.DeviceArray.from_host(cfg["phi"])
        dF = gpu.DeviceArray.from_host(cfg["F"])
        ws.normal(d, dF, fb, cfg["dx"], cfl=0.5, nsteps=3, reinit_interval=10 ** 9,
                  reinit_iters=0, use_phi0=0)
        ws.reinit(d, fb, cfg["dx"], cfl=0.5, iters=2, use_phi0=0)
        got = d.download()
    finally:
        integrator.set_fp_mode(prev)
    g = Grid(cfg["n"], dx=cfg["dx"])
    phi = g.field(cfg["phi"])
    ps = PatchedNormalStepper(oracle.oracle_toolbox(), g, os.cpu_count() or 1)
    parts, Fs = ps.scatter(phi), ps.scatter(g.field(cfg["F"]))
    for _ in range(3):
        ps.normal_step(parts, Fs, 0.5)
    ps.reinit(parts, 0.5, 2, 0)
    ps.gather(parts, phi)
    assert rel_err(g.interior(g.field(got)), g.interior(phi)) <= REL_FAST


@pytest.mark.parametrize("use0", [0, 1])
def test_reinitialization(mode, use0):
    from lsmlib_b200 import gpu, integrator
    g = Grid((26, 22, 30), dx=(0.05, 0.05, 0.05))
    phi0 = 3.0 * spheres(g, (-0.6, -0.6, -0.6), seed=5, count=3)   # not a distance
    st = Stepper(oracle.oracle_toolbox(), g)
    ref = g.field(phi0)
    st.reinit(ref, 0.5, 4, use0=use0)
    ws = integrator.Workspace(g.gb, 8)
    d = gpu.DeviceArray.from_host(phi0)
    ws.reinit(d, g.fb, g.dx, cfl=0.5, iters=4, use_phi0=use0)
    check(mode, g.interior(g.field(d.download())), g.interior(ref))


def test_deformation_field_matches_oracle():
    """LeVeque's field is evaluated on the device (CUDA sin/cos) and on the
    host (numpy); the two differ by a few ulps, so the comparison is at the
    fast-mode tolerance."""
    from lsmlib_b200 import gpu, integrator
    n = (40, 40, 40)
    g = Grid(n, dx=(1.0 / 40,) * 3)
    x_lo = (0.0, 0.0, 0.0)
    phi0 = sphere(g, x_lo, c=(0.35, 0.35, 0.35), r=0.15)
    st = Stepper(oracle.oracle_toolbox(), g)
    ref = g.field(phi0)
    t = 0.0
    for _ in range(3):
        v0 = deformation_velocity(g, x_lo, t)
        dt = st.advect_dt(v0, 0.5)
        st.advect_step(ref, lambda c: deformation_velocity(g, x_lo, t + c * dt), dt)
        t += dt
    ws = integrator.Workspace(g.gb, 8)
    d = gpu.DeviceArray.from_host(phi0)
    ws.deformation(d, g.fb, g.dx, x_lo, period=3.0, cfl=0.5, t_end=3.0, nsteps=3)
    tg, _ = ws.time()
    assert abs(tg - t) <= 1e-12 * t
    assert rel_err(g.interior(g.field(d.download())), g.interior(ref)) <= REL_FAST


def test_single_stage_with_caller_ghosts(mode):
    """bc_mask = 0: the stage reads the ghost cells stored in phi_s (a patch
    whose halo came from a neighbour), on a fill box with non-zero bounds."""
    from lsmlib_b200 import gpu, integrator
    rng = np.random.default_rng(2)
    g = Grid((21, 14, 12), lo=(-5, 3, 7), dx=(0.1, 0.1, 0.1))
    phi = g.field(rng.standard_normal(g.shape))
    vel = [g.field(rng.standard_normal(g.shape)) for _ in range(3)]
    tb = oracle.oracle_toolbox()
    st = Stepper(tb, g)
    st.zero_rhs()
    f = dict(st.up)
    f.update({"phi": phi, "vel_x": vel[0], "vel_y": vel[1], "vel_z": vel[2]})
    tb.call("lsm3dupwindhjweno5_", f, g.fb, **g.dxyz())
    tb.call("lsm3daddadvectiontermtolserhs_",
            {"lse_rhs": st.rhs, "phi_x": st.up["phi_x"], "phi_y": st.up["phi_y"],
             "phi_z": st.up["phi_z"], "vel_x": vel[0], "vel_y": vel[1],
             "vel_z": vel[2]}, g.fb)
    out = g.zeros()
    tb.call("lsm3dtvdrk3stage1_", {"u_stage1": out, "u_cur": phi, "rhs": st.rhs},
            g.fb, dt=0.013)
    d_out = gpu.DeviceArray(g.shape)
    d_phi = gpu.DeviceArray.from_host(phi.data)
    dv = [gpu.DeviceArray.from_host(v.data) for v in vel]
    integrator.stage(0, 8, d_out, d_phi, d_phi, dv, g.gb, g.fb, g.dx, 0.013, 1,
                     bc_mask=0)
    check(mode, g.interior(g.field(d_out.download())), g.interior(out))


FP32_POLICIES = [None, 0, 1, 4, 7]   # None: the workspace default (sign | SR)


def fp32_normal_run(policy):
    """10 normal-velocity steps with a reinitialization every 5 steps on a
    48^3 union of spheres; the FP32 workspace result and the FP64 oracle's."""
    from lsmlib_b200 import gpu, integrator
    n = (48, 48, 48)
    g = Grid(n, dx=(2.0 / 48,) * 3)
    x_lo = (-1.0, -1.0, -1.0)
    phi0 = spheres(g, x_lo, seed=11)
    x, y, z = g.centers(x_lo)
    F = 1.0 + 0.2 * np.sin(4 * np.pi * x) * np.sin(4 * np.pi * y) * np.sin(4 * np.pi * z)
    st = Stepper(oracle.oracle_toolbox(), g)
    ref = g.field(phi0)
    Ff = g.field(F)
    for s in range(10):
        st.normal_step(ref, Ff, 0.5)
        if (s + 1) % 5 == 0:
            st.reinit(ref, 0.5, 4)
    ws = integrator.Workspace(g.gb, 4)
    if policy is not None:
        ws.set_fp64_policy(policy)
    d = gpu.DeviceArray.from_host(phi0.astype(np.float32))
    dF = gpu.DeviceArray.from_host(F.astype(np.float32))
    ws.normal(d, dF, g.fb, g.dx, cfl=0.5, nsteps=10, reinit_interval=5,
              reinit_iters=4)
    got = g.interior(g.field(d.download().astype(np.float64)))
    return got, g.interior(ref)


@pytest.mark.parametrize("policy", FP32_POLICIES)
def test_fp32_form_error_against_fp64(policy):
    """FP32 storage and arithmetic (FP64 CFL reduction, dt and t) under each
    FP64 policy (kink stencils in FP64, smoothed sign in FP64, stochastic
    rounding of the stage outputs) stays within 1e-5 of the FP64 oracle."""
    got, want = fp32_normal_run(policy)
    err = np.abs(got - want)
    assert err.max() <= ABS_FP32, err.max()


def test_fp32_stochastic_rounding_is_reproducible_and_unbiased():
    """Two fresh workspaces draw the same seeds (bit-identical results), and
    the mean error of the stochastically rounded run is below the
    round-to-nearest run's."""
    from lsmlib_b200 import integrator
    a, want = fp32_normal_run(integrator.STOCH_ROUND)
    b, _ = fp32_normal_run(integrator.STOCH_ROUND)
    assert same_bits(a, b)
    rn, _ = fp32_normal_run(0)
    assert np.mean(np.abs(a - want)) < np.mean(np.abs(rn - want))


@pytest.mark.parametrize("bc", ["copy", "periodic"])
def test_generated_boundary_kinds(mode, bc):
    """Copy extrapolation (homogeneous Neumann) and periodic ghost values are
    generated on the fly like the linear ones."""
    from lsmlib_b200 import gpu, integrator
    rng = np.random.default_rng(21)
    g = Grid((30, 19, 26), dx=(0.07, 0.06, 0.08))
    phi0 = spheres(g, (-1.0, -0.6, -1.0), seed=9, count=4)
    vel = [g.field(np.full(g.shape, c)) for c in rng.uniform(-1, 1, 3)]
    st = Stepper(oracle.oracle_toolbox(), g, bc=bc)
    ref = g.field(phi0)
    dt = st.advect_dt(vel, 0.5)
    for _ in range(3):
        st.advect_step(ref, lambda c: vel, dt)
    ws = integrator.Workspace(g.gb, 8)
    ws.set_bc(integrator.BC_COPY if bc == "copy" else integrator.BC_PERIODIC)
    d = gpu.DeviceArray.from_host(phi0)
    dv = [gpu.DeviceArray.from_host(v.data) for v in vel]
    ws.advect(d, dv, g.fb, g.dx, cfl=0.5, nsteps=3)
    check(mode, g.interior(g.field(d.download())), g.interior(ref))


def test_config1_full_run_strict_matches_oracle():
    """The reference's CPU-runnable case end to end: 64^3 on [-1,1]^3, sphere
    r = 0.25 at (0.1,-0.05,0), velocity (1, 0.5, 0.25) stored as arrays, CFL
    0.5, 100 TVD-RK3 steps with linear-extrapolation ghosts -- strict GPU
    arithmetic equals the oracle's reference-order chain bit for bit."""
    from lsmlib_b200 import gpu, integrator, workloads
    cfg = workloads.config1()
    g = Grid(cfg["n"], dx=cfg["dx"])
    vel = [g.field(v) for v in cfg["vel"]]
    st = Stepper(oracle.oracle_toolbox(), g)
    ref = g.field(cfg["phi"].copy(order="F"))  # the oracle steps in place
    dt = st.advect_dt(vel, cfg["cfl"])
    for _ in range(cfg["steps"]):
        st.advect_step(ref, lambda c: vel, dt)
    prev = integrator.get_fp_mode()
    integrator.set_fp_mode(integrator.FP_STRICT)
    try:
        ws = integrator.Workspace(g.gb, 8)
        d = gpu.DeviceArray.from_host(cfg["phi"])
        dv = [gpu.DeviceArray.from_host(v) for v in cfg["vel"]]
        ws.advect(d, dv, g.fb, g.dx, cfl=cfg["cfl"], nsteps=cfg["steps"])
        got = g.interior(g.field(d.download()))
    finally:
        integrator.set_fp_mode(prev)
    assert same_bits(got, g.interior(ref))


@pytest.mark.parametrize("n", [(37, 11, 70), (64, 40, 33), (20, 20, 17)])
@pytest.mark.parametrize("steps,interval", [(1, 0), (3, 2), (2, 2)])
def test_normal_host_buffers_match_device_driver(mode, n, steps, interval):
    """lsmgpu_normal_tvdrk3_host (host phi and F, slab-pipelined copies) gives
    the device driver's values bit for bit, with and without a
    reinitialization after the last step."""
    from lsmlib_b200 import gpu, integrator
    g = Grid(n, dx=(2.0 / n[0],) * 3)
    x_lo = (-1.0, -1.0, -1.0)
    phi0 = np.asfortranarray(spheres(g, x_lo, seed=5))
    x, y, z = g.centers(x_lo)
    F = np.asfortranarray(1.0 + 0.2 * np.sin(4 * np.pi * x) * np.sin(4 * np.pi * y) *
                          np.sin(4 * np.pi * z))
    ws = integrator.Workspace(g.gb, 8)
    d = gpu.DeviceArray.from_host(phi0)
    dF = gpu.DeviceArray.from_host(F)
    ws.normal(d, dF, g.fb, g.dx, cfl=0.5, nsteps=steps, reinit_interval=interval,
              reinit_iters=3)
    want = d.download()
    ws2 = integrator.Workspace(g.gb, 8)
    host = phi0.copy(order="F")
    ws2.normal_host(host, F, g.fb, g.dx, cfl=0.5, nsteps=steps, reinit_interval=interval,
                    reinit_iters=3)
    assert same_bits(host, want)
    # a second call continues from the host state, as two device calls would
    ws.normal(d, dF, g.fb, g.dx, cfl=0.5, nsteps=1, step0=steps)
    ws2.normal_host(host, F, g.fb, g.dx, cfl=0.5, nsteps=1, step0=steps)
    assert same_bits(host, d.download())
    ws.close()
    ws2.close()


def test_queued_host_calls_match_device_driver(mode):
    """lsmgpu_workspace_set_host_async(ws, 1): one-step host calls queued back
    to back on pinned phi and F (each call's slabs copied in behind the
    previous call's copies back, the speed in alternating device buffers),
    a reinitialization every other step, then lsmgpu_workspace_sync: the
    device driver's values bit for bit."""
    import ctypes

    from lsmlib_b200 import gpu, integrator
    n = (48, 40, 70)
    g = Grid(n, dx=(2.0 / n[0],) * 3)
    x_lo = (-1.0, -1.0, -1.0)
    phi0 = np.asfortranarray(spheres(g, x_lo, seed=9))
    x, y, z = g.centers(x_lo)
    F = np.asfortranarray(1.0 + 0.2 * np.sin(4 * np.pi * x) * np.sin(4 * np.pi * y) *
                          np.sin(4 * np.pi * z))
    steps = 5
    ws = integrator.Workspace(g.gb, 8)
    d = gpu.DeviceArray.from_host(phi0)
    dF = gpu.DeviceArray.from_host(F)
    ws.normal(d, dF, g.fb, g.dx, cfl=0.5, nsteps=steps, reinit_interval=2, reinit_iters=2)
    want = d.download()
    lib = gpu.load()
    hp_addr = lib.lsmgpu_host_alloc(phi0.nbytes)
    hf_addr = lib.lsmgpu_host_alloc(F.nbytes)
    try:
        count = phi0.size
        hp = np.ctypeslib.as_array((ctypes.c_double * count).from_address(hp_addr))
        hf = np.ctypeslib.as_array((ctypes.c_double * count).from_address(hf_addr))
        hp[:] = phi0.ravel(order="F")
        hf[:] = F.ravel(order="F")
        ws2 = integrator.Workspace(g.gb, 8)
        ws2.set_host_async(True)
        for s in range(steps):
            ws2.normal_host(hp_addr, hf_addr, g.fb, g.dx, cfl=0.5, nsteps=1, step0=s,
                            reinit_interval=2, reinit_iters=2)
        ws2.sync()
        got = hp.reshape(phi0.shape, order="F").copy(order="F")
        assert same_bits(got, want)
        ws2.close()
    finally:
        lib.lsmgpu_host_free(hp_addr)
        lib.lsmgpu_host_free(hf_addr)
    ws.close()
