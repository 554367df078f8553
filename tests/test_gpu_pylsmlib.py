"""pylsmlib.LevelSetIntegrator on torch tensors runs the same kernels as the
Workspace drivers (themselves pinned to the oracle): bit-identical results for
normal speed with reinitialization, external velocity, the deformation field
and reinitialization alone, FP64 and FP32, on a non-default torch stream."""
import numpy as np
import pytest
import torch

from lsmlib_b200 import gpu, integrator
from pylsmlib import Grid, LevelSetIntegrator

pytestmark = pytest.mark.gpu


def as_fortran(t):
    """(nz, ny, nx) C-ordered tensor -> (nx, ny, nz) Fortran-ordered array."""
    return np.asfortranarray(t.detach().cpu().numpy().T)


def setup(dtype):
    g = Grid.set_grid_dims((30, 22, 17), (-1.0, -0.8, -0.7), (1.0, 0.8, 0.7))
    x, y, z = g.coordinates(dtype=torch.float64)
    phi = torch.minimum(torch.sqrt((x - 0.2) ** 2 + y ** 2 + z ** 2) - 0.45,
                        torch.sqrt((x + 0.4) ** 2 + (y - 0.2) ** 2 + z ** 2) - 0.3)
    F = 1.0 + 0.3 * torch.sin(3 * x) * torch.cos(2 * y)
    vel = (0.8 + 0.1 * y, -0.5 + 0.2 * z, 0.3 * torch.cos(x))
    cast = lambda t: t.to(dtype).contiguous()
    return g, cast(phi), cast(F), [cast(v) for v in vel]


def workspace_run(g, prec, what, phi, F=None, vel=None):
    ws = integrator.Workspace(g.gb, prec)
    d = gpu.DeviceArray.from_host(as_fortran(phi))
    if what == "normal":
        dF = gpu.DeviceArray.from_host(as_fortran(F))
        ws.normal(d, dF, g.fb, g.dx, cfl=0.5, nsteps=4, step0=0, reinit_interval=2,
                  reinit_iters=3)
    elif what == "external":
        dv = [gpu.DeviceArray.from_host(as_fortran(v)) for v in vel]
        ws.advect(d, dv, g.fb, g.dx, cfl=0.5, nsteps=3)
    elif what == "deformation":
        x_lo = tuple(g.x_lo_ghostbox[k] - 0.5 * g.dx[k] for k in range(3))
        ws.deformation(d, g.fb, g.dx, x_lo, period=3.0, cfl=0.5, t_end=3.0, nsteps=3)
    else:
        ws.reinit(d, g.fb, g.dx, cfl=0.5, iters=5)
    out = d.download()
    t, dt = ws.time()
    return out, t


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("what", ["normal", "external", "deformation", "reinit"])
def test_front_door_matches_workspace_drivers(dtype, what):
    prev = integrator.get_fp_mode()
    g, phi, F, vel = setup(dtype)
    prec = 8 if dtype == torch.float64 else 4
    integrator.set_fp_mode(integrator.FP_FAST)
    want, t_want = workspace_run(g, prec, what, phi, F, vel)
    integ = LevelSetIntegrator(g, dtype=dtype, reinit_interval=2, reinit_iters=3)
    s = torch.cuda.Stream()
    p = phi.clone()
    with torch.cuda.stream(s):
        if what == "normal":
            integ.advance_normal(p, F, nsteps=4)
        elif what == "external":
            integ.advance_external(p, vel, nsteps=3)
        elif what == "deformation":
            integ.advance_deformation(p, period=3.0, t_end=3.0, nsteps=3)
        else:
            integ.reinitialize(p, iters=5)
    s.synchronize()
    gpu.check_rc(gpu.load().lsmgpu_set_stream(None), "set_stream")
    integrator.set_fp_mode(prev)
    got = as_fortran(p)
    view = np.uint64 if dtype == torch.float64 else np.uint32
    lo, hi = (g.ilo_fb, g.jlo_fb, g.klo_fb), (g.ihi_fb, g.jhi_fb, g.khi_fb)
    sl = tuple(slice(a, b + 1) for a, b in zip(lo, hi))
    assert np.array_equal(np.ascontiguousarray(got[sl]).view(view),
                          np.ascontiguousarray(want[sl]).view(view))
    if what != "reinit":
        assert integ.time[0] == t_want
    integ.close()


def test_rejects_wrong_tensors():
    g, phi, F, vel = setup(torch.float64)
    integ = LevelSetIntegrator(g)
    with pytest.raises(ValueError):
        integ.advance_normal(phi.float(), F)           # wrong dtype
    with pytest.raises(ValueError):
        integ.advance_normal(phi.cpu(), F)             # host tensor
    with pytest.raises(ValueError):
        integ.advance_normal(phi[:, :, :-1], F)        # wrong shape
    integ.close()
