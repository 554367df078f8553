"""The FP64 band form of an FP32 workspace (policy FP64_BAND) on the
deformation driver, fast mode.

Tiles within the band of the interface are computed in FP64 from FP64 copies
of the stage arrays, the others in FP32, and every cell is written in both
precisions.  With every tile in the band the result must be the FP64 run's,
rounded to FP32, bit for bit; with the default band the error against the
FP64 run near the interface must fall below the plain FP32 form's."""
import numpy as np
import pytest

from oracle.driver import Grid

pytestmark = pytest.mark.gpu


@pytest.fixture
def fast():
    from lsmlib_b200 import integrator
    prev = integrator.get_fp_mode()
    integrator.set_fp_mode(integrator.FP_FAST)
    yield
    integrator.set_fp_mode(prev)


def sphere(g, c=(0.35, 0.35, 0.35), r=0.15):
    x, y, z = g.centers((0.0, 0.0, 0.0))
    return np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - r


def run(g, phi0, precision, chunks, band_cells=None, ws=None, d=None):
    """Deformation steps in calls of chunks[i] steps; the workspace, the
    device level set and the interior of the result as float64."""
    from lsmlib_b200 import gpu, integrator
    if ws is None:
        ws = integrator.Workspace(g.gb, precision)
        if band_cells is not None:
            ws.set_fp64_policy(integrator.FP64_SIGN | integrator.STOCH_ROUND
                               | integrator.FP64_BAND)
            ws.set_fp64_band(band_cells)
    if d is None:
        d = gpu.DeviceArray.from_host(phi0.astype(np.float64 if precision == 8 else np.float32))
    for n in chunks:
        ws.deformation(d, g.fb, g.dx, (0.0, 0.0, 0.0), period=3.0, cfl=0.5, t_end=3.0,
                       nsteps=n)
    return ws, d, g.interior(g.field(d.download().astype(np.float64)))


def as_f32_bits(a):
    return np.ascontiguousarray(a.astype(np.float32)).view(np.uint32)


@pytest.mark.parametrize("n", [(64, 56, 48), (70, 33, 37)])
def test_every_tile_in_fp64_is_the_fp64_run_rounded(fast, n):
    """band half-width 1e6 cells: every tile in FP64.  Three calls (the FP64
    copy of phi carried between them) against one FP64 workspace from the
    same FP32-rounded start: equal after rounding, bit for bit, with the
    same time."""
    g = Grid(n, dx=(1.0 / 64,) * 3)
    phi0 = sphere(g).astype(np.float32).astype(np.float64)
    ws64, _, want = run(g, phi0, 8, [24])
    ws32, _, got = run(g, phi0, 4, [8, 8, 8], band_cells=1e6)
    assert np.array_equal(as_f32_bits(got), as_f32_bits(want)), \
        np.max(np.abs(got - want))
    assert ws32.time() == ws64.time()


def test_caller_changes_to_phi_reload_the_fp64_copy(fast):
    """After a call, the caller writes a new level set into phi: the next
    call starts from it (the FP64 copy is reloaded wherever it no longer
    rounds to phi), as a fresh workspace would."""
    g = Grid((48, 40, 40), dx=(1.0 / 48,) * 3)
    first = sphere(g)
    second = sphere(g, c=(0.5, 0.45, 0.4), r=0.2).astype(np.float32).astype(np.float64)
    ws, d, _ = run(g, first, 4, [6], band_cells=1e6)
    d.upload(second)
    ws.set_time(0.0)
    _, _, got = run(g, None, 4, [6], ws=ws, d=d)
    _, _, want = run(g, second, 8, [6])
    assert np.array_equal(as_f32_bits(got), as_f32_bits(want)), \
        np.max(np.abs(got - want))


def test_default_band_is_closer_to_fp64_than_plain_fp32(fast):
    """120 steps at 64^3: in the band |phi| < 5 dx of the FP64 run the band
    form's error against FP64 is below the plain FP32 form's (both with the
    default stochastic rounding), and within 1e-6."""
    g = Grid((64, 64, 64), dx=(1.0 / 64,) * 3)
    phi0 = sphere(g).astype(np.float32).astype(np.float64)
    chunks = [40, 40, 40]
    _, _, want = run(g, phi0, 8, chunks)
    _, _, plain = run(g, phi0, 4, chunks)
    _, _, band = run(g, phi0, 4, chunks, band_cells=16.0)
    near = np.abs(want) < 5 * g.dx[0]
    e_plain = np.abs(plain - want)[near].max()
    e_band = np.abs(band - want)[near].max()
    assert e_band < e_plain, (e_band, e_plain)
    assert e_band <= 1e-6, e_band
