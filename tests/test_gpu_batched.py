"""Batched grids: one persistent work-list launch per TVD-RK3 stage.

Every grid of a small uneven batch must match the oracle's reference-order
chain for its own constant velocity and CFL dt (fast arithmetic: 1e-12
relative); graph replay, plain persistent launches and per-grid launches must
agree bit for bit; the autotuner must leave the state untouched; the FP32
batch must stay within 1e-5 of the FP64 batch."""
import numpy as np
import pytest

import oracle
from oracle.driver import Grid, Stepper

pytestmark = pytest.mark.gpu


def small_batch(seed=3, ngrids=7):
    from lsmlib_b200 import workloads
    return workloads.config4(ngrids=ngrids, seed=seed, lo_n=9, hi_n=41)


def test_batched_matches_oracle_per_grid():
    from lsmlib_b200 import batched, workloads
    cfg = small_batch()
    phis = workloads.config4_phi(cfg)
    b = batched.Batch(cfg["sizes"], cfg["dx"], 8)
    b.upload(phis)
    b.set_velocity(cfg["vel"], 0.5)
    dts = b.dt()
    b.advect(3, batched.MODE_GRAPH)
    got = b.download()
    orc = oracle.oracle_toolbox()
    for g, (n, dx, v) in enumerate(zip(cfg["sizes"], cfg["dx"], cfg["vel"])):
        grid = Grid(n, dx=dx)
        phi = grid.field(phis[g])
        vel = [grid.field(np.full(grid.shape, c)) for c in v]
        st = Stepper(orc, grid)
        assert dts[g] == st.advect_dt(vel, 0.5)
        for _ in range(3):
            st.advect_step(phi, lambda c: vel, dts[g])
        want = grid.interior(phi)
        have = grid.interior(grid.field(got[g]))
        assert np.max(np.abs(have - want)) <= 1e-12 * np.max(np.abs(want)), g


def test_launch_modes_agree_bitwise():
    from lsmlib_b200 import batched, workloads
    cfg = small_batch(seed=5, ngrids=9)
    phis = workloads.config4_phi(cfg)
    outs = []
    for mode in (batched.MODE_GRAPH, batched.MODE_PERSISTENT, batched.MODE_PER_GRID):
        b = batched.Batch(cfg["sizes"], cfg["dx"], 8)
        b.upload(phis)
        b.set_velocity(cfg["vel"], 0.5)
        b.advect(2, mode)
        outs.append(np.concatenate([a.ravel() for a in b.download()]))
        b.close()
    assert np.array_equal(outs[0].view(np.uint64), outs[1].view(np.uint64))
    assert np.array_equal(outs[0].view(np.uint64), outs[2].view(np.uint64))


@pytest.mark.parametrize("shape", range(15))
@pytest.mark.parametrize("prec", [8, 4])
def test_every_tile_shape_gives_the_same_result(shape, prec):
    """Every tile shape and halo-staging schedule (one cell per thread with a
    shared plane or direct loads, two cells per thread) gives the same bits,
    in FP64 and in FP32 with stochastic rounding and FP64 kinks."""
    from lsmlib_b200 import batched, workloads
    cfg = small_batch(seed=8, ngrids=5)
    dtype = np.float64 if prec == 8 else np.float32
    phis = workloads.config4_phi(cfg, dtype)
    res = []
    for s in (1, shape):
        b = batched.Batch(cfg["sizes"], cfg["dx"], prec)
        b.upload(phis)
        b.set_velocity(cfg["vel"], 0.5)
        if prec == 4:
            b.set_fp64_policy(5)
        b.set_tile(s)
        b.advect(2, batched.MODE_PERSISTENT)
        res.append(np.concatenate([a.ravel() for a in b.download()]))
    u = np.uint64 if prec == 8 else np.uint32
    assert np.array_equal(res[0].view(u), res[1].view(u))


@pytest.mark.parametrize("shape", [10, 11, 12, 13, 14])
def test_fp32_packed_schedule_matches_one_cell_per_thread(shape):
    """FP32 without the FP64 kink recomputation: the two-cells-per-thread
    schedule evaluates both cells' WENO5 sides as one packed FP32x2
    computation, which rounds differently from the scalar one-cell schedule;
    the two stay within a few FP32 ulps of the level set's scale."""
    from lsmlib_b200 import batched, workloads
    cfg = small_batch(seed=8, ngrids=5)
    phis = workloads.config4_phi(cfg, np.float32)
    res = []
    for s in (0, shape):
        b = batched.Batch(cfg["sizes"], cfg["dx"], 4)
        b.upload(phis)
        b.set_velocity(cfg["vel"], 0.5)
        b.set_fp64_policy(0)
        b.set_tile(s)
        b.advect(2, batched.MODE_PERSISTENT)
        res.append(np.concatenate([a.ravel() for a in b.download()]).astype(np.float64))
    scale = np.max(np.abs(res[0]))
    assert np.max(np.abs(res[0] - res[1])) <= 1e-5 * scale


def test_autotune_keeps_state_and_picks_a_shape():
    from lsmlib_b200 import batched, workloads
    cfg = small_batch(seed=11, ngrids=6)
    phis = workloads.config4_phi(cfg)
    b = batched.Batch(cfg["sizes"], cfg["dx"], 8)
    b.upload(phis)
    b.set_velocity(cfg["vel"], 0.5)
    before = np.concatenate([a.ravel() for a in b.download()])
    ms = b.autotune(report=True)
    assert all(t > 0 for t in ms)
    after = np.concatenate([a.ravel() for a in b.download()])
    assert np.array_equal(before, after)
    s, tile = b.tile()
    assert 0 <= s < 15 and tile[1] == 8


def test_fp32_batch_error_against_fp64():
    from lsmlib_b200 import batched, workloads
    cfg = small_batch(seed=13, ngrids=6)
    res = {}
    for prec in (8, 4):
        dt = np.float64 if prec == 8 else np.float32
        b = batched.Batch(cfg["sizes"], cfg["dx"], prec)
        b.upload(workloads.config4_phi(cfg, dt))
        b.set_velocity(cfg["vel"], 0.5)
        b.advect(10, batched.MODE_GRAPH)
        res[prec] = np.concatenate([a[3:-3, 3:-3, 3:-3].ravel().astype(np.float64)
                                    for a in b.download()])
    assert np.max(np.abs(res[4] - res[8])) <= 1e-5


@pytest.mark.parametrize("bc", [1, 2])
def test_batched_copy_and_periodic_boundaries(bc):
    from lsmlib_b200 import batched, workloads
    cfg = small_batch(seed=17, ngrids=4)
    phis = workloads.config4_phi(cfg)
    b = batched.Batch(cfg["sizes"], cfg["dx"], 8)
    b.upload(phis)
    b.set_velocity(cfg["vel"], 0.5)
    b.set_bc(bc)
    dts = b.dt()
    b.advect(2, batched.MODE_GRAPH)
    got = b.download()
    for g, (n, dx, v) in enumerate(zip(cfg["sizes"], cfg["dx"], cfg["vel"])):
        grid = Grid(n, dx=dx)
        phi = grid.field(phis[g])
        vel = [grid.field(np.full(grid.shape, c)) for c in v]
        st = Stepper(oracle.oracle_toolbox(), grid, bc="copy" if bc == 1 else "periodic")
        for _ in range(2):
            st.advect_step(phi, lambda c: vel, dts[g])
        want = grid.interior(phi)
        have = grid.interior(grid.field(got[g]))
        assert np.max(np.abs(have - want)) <= 1e-12 * np.max(np.abs(want)), g
