"""Python front end of the fused TVD-RK3 drivers of liblsmgpu.so.

``Workspace(gb, precision)`` owns the device stage buffers of one grid; its
methods advance a device-resident level set (a
:class:`lsmlib_b200.gpu.DeviceArray` with the workspace's ghost box):

* ``advect(phi, vel, fb, dx, cfl, dt_fixed, t_end, nsteps)`` -- external
  velocity arrays (the reference's advection integrator);
* ``deformation(phi, fb, dx, x_lo, period, cfl, t_end, nsteps)`` -- LeVeque's
  time-reversing deformation field evaluated on the device;
* ``normal(phi, F, fb, dx, cfl, nsteps, ...)`` -- normal-velocity motion with
  periodic reinitialization;
* ``reinit(phi, fb, dx, cfl, iters, use_phi0)``.
"""
import ctypes

import numpy as np

from . import gpu
from .ext_abi import dbls, ints

FP_STRICT, FP_FAST = 0, 1
# boundary masks (per face f = x-lo .. z-hi): linear, copy, periodic
BC_LINEAR, BC_COPY, BC_PERIODIC = 0x3F, 0x3F << 8, 0x3F << 16
# FP64 parts of the FP32 form (Workspace.set_fp64_policy): kink stencils in
# FP64, reinitialization sign in FP64, stochastic rounding of stage outputs,
# the tiles near the interface in FP64 (deformation driver, fast mode)
FP64_KINKS, FP64_SIGN, STOCH_ROUND, FP64_BAND = 1, 2, 4, 8


def set_fp_mode(mode):
    gpu.check_rc(gpu.load().lsmgpu_set_fp_mode(int(mode)), "set_fp_mode")


def get_fp_mode():
    return gpu.load().lsmgpu_get_fp_mode()


class Workspace:
    def __init__(self, gb, precision=8):
        lib = gpu.load()
        self.gb = tuple(int(v) for v in gb)
        self.precision = int(precision)
        h = ctypes.c_void_p()
        gpu.check_rc(lib.lsmgpu_workspace_create(ctypes.byref(h), ints(self.gb),
                                                 self.precision), "workspace_create")
        self.h = h

    def close(self):
        if self.h:
            gpu.load().lsmgpu_workspace_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_bc(self, mask):
        gpu.check_rc(gpu.load().lsmgpu_workspace_set_bc(self.h, int(mask)), "set_bc")

    def set_host_async(self, on):
        """Queue normal_host calls instead of waiting for each (see
        lsmgpu_workspace_set_host_async); sync() waits for them."""
        gpu.check_rc(gpu.load().lsmgpu_workspace_set_host_async(self.h, int(bool(on))),
                     "set_host_async")

    def sync(self):
        gpu.check_rc(gpu.load().lsmgpu_workspace_sync(self.h), "workspace_sync")

    def set_fp64_policy(self, policy):
        """FP32 workspaces: FP64_KINKS | FP64_SIGN | STOCH_ROUND | FP64_BAND."""
        gpu.check_rc(gpu.load().lsmgpu_workspace_set_fp64_policy(self.h, int(policy)),
                     "set_fp64_policy")

    def set_fp64_band(self, cells, widen=1):
        """Half-width in cells of the FP64 band (FP64_BAND): tiles holding a
        cell with |phi| < cells * min(dx), and their neighbours when widen
        is 1, run in FP64."""
        gpu.check_rc(gpu.load().lsmgpu_workspace_set_fp64_band(self.h, float(cells),
                                                               int(widen)),
                     "set_fp64_band")

    def set_time(self, t):
        gpu.check_rc(gpu.load().lsmgpu_workspace_set_time(self.h, float(t)), "set_time")

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        gpu.check_rc(gpu.load().lsmgpu_workspace_get_time(self.h, ctypes.byref(t),
                                                          ctypes.byref(dt)), "get_time")
        return t.value, dt.value

    def advect(self, phi, vel, fb, dx, cfl=0.5, dt_fixed=0.0, t_end=0.0, nsteps=1):
        rc = gpu.load().lsmgpu_advect_tvdrk3(self.h, phi.ptr, vel[0].ptr, vel[1].ptr,
                                             vel[2].ptr, ints(fb), dbls(dx), cfl,
                                             dt_fixed, t_end, int(nsteps))
        gpu.check_rc(rc, "advect_tvdrk3")

    def deformation(self, phi, fb, dx, x_lo, period=3.0, cfl=0.5, t_end=3.0,
                    nsteps=1):
        rc = gpu.load().lsmgpu_deformation_tvdrk3(self.h, phi.ptr, ints(fb), dbls(dx),
                                                  dbls(x_lo), period, cfl, t_end,
                                                  int(nsteps))
        gpu.check_rc(rc, "deformation_tvdrk3")

    def normal(self, phi, F, fb, dx, cfl=0.5, nsteps=1, step0=0,
               reinit_interval=0, reinit_iters=0, use_phi0=0):
        rc = gpu.load().lsmgpu_normal_tvdrk3(self.h, phi.ptr, F.ptr, ints(fb),
                                             dbls(dx), cfl, int(nsteps), int(step0),
                                             int(reinit_interval), int(reinit_iters),
                                             int(use_phi0))
        gpu.check_rc(rc, "normal_tvdrk3")

    def normal_host(self, phi, F, fb, dx, cfl=0.5, nsteps=1, step0=0,
                    reinit_interval=0, reinit_iters=0, use_phi0=0):
        """``normal`` on host arrays (numpy, Fortran order, the workspace's
        ghost box, or raw host addresses); phi is updated in place."""
        def addr(a):
            return a.ctypes.data if hasattr(a, "ctypes") else int(a)
        rc = gpu.load().lsmgpu_normal_tvdrk3_host(self.h, addr(phi), addr(F), ints(fb),
                                                  dbls(dx), cfl, int(nsteps), int(step0),
                                                  int(reinit_interval), int(reinit_iters),
                                                  int(use_phi0))
        gpu.check_rc(rc, "normal_tvdrk3_host")

    def reinit(self, phi, fb, dx, cfl=0.5, iters=1, use_phi0=0):
        rc = gpu.load().lsmgpu_reinit_tvdrk3(self.h, phi.ptr, ints(fb), dbls(dx), cfl,
                                             int(iters), int(use_phi0))
        gpu.check_rc(rc, "reinit_tvdrk3")


def stage(kind, precision, out, phi_s, phi_n, aux, gb, fb, dx, dt, rk_kind,
          bc_mask=0x3f, dom=None, dt_dev=None, use_phi0=0):
    """One fused stage (lsmgpu_lse_stage) on device arrays."""
    a = [x.ptr if x is not None else None for x in (list(aux) + [None] * 3)[:3]]
    rc = gpu.load().lsmgpu_lse_stage(int(kind), int(precision), out.ptr, phi_s.ptr,
                                     phi_n.ptr if phi_n is not None else None,
                                     a[0], a[1], a[2], ints(gb), ints(fb),
                                     ints(dom) if dom is not None else None,
                                     int(bc_mask), dbls(dx), dt_dev, float(dt),
                                     int(rk_kind), int(use_phi0))
    gpu.check_rc(rc, "lse_stage")
