"""Python front end of the discrete adjoint (lsmgpu_adjoint_* of liblsmgpu.so).

``AdvectionAdjoint(n, dx, x_lo, lattice, nsteps, checkpoint_every)`` owns one
problem: upwind WENO5 + TVD-RK3 advection of phi by a trilinear B-spline
velocity (coefficients theta[3][m][m][m], x fastest), frozen dt, loss
sum (H(phi_T) - H(target))^2 dx dy dz.  ``forward()`` returns the loss and
keeps the checkpoints; ``backward(seed)`` returns seed * dJ/dtheta and
seed * dJ/dphi0.
"""
import ctypes

import numpy as np

from . import gpu
from .ext_abi import dbls, ints


class AdvectionAdjoint:
    def __init__(self, n, dx, x_lo, lattice=8, nsteps=200, checkpoint_every=15):
        lib = gpu.load()
        self.n = tuple(int(v) for v in n)
        self.lattice = int(lattice)
        self.shape = tuple(v + 6 for v in self.n)
        h = ctypes.c_void_p()
        gpu.check_rc(lib.lsmgpu_adjoint_create(ctypes.byref(h), ints(self.n), dbls(dx),
                                               dbls(x_lo), self.lattice, int(nsteps),
                                               int(checkpoint_every)), "adjoint_create")
        self.h = h

    def close(self):
        if self.h:
            gpu.load().lsmgpu_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_theta(self, theta):
        t = np.ascontiguousarray(np.asarray(theta, dtype=np.float64).reshape(
            3, self.lattice, self.lattice, self.lattice))
        # x fastest: theta[d][z][y][x] in C order
        self._theta = t
        gpu.check_rc(gpu.load().lsmgpu_adjoint_set_theta(self.h, t.ctypes.data), "set_theta")

    def cfl_dt(self, cfl):
        v = ctypes.c_double()
        gpu.check_rc(gpu.load().lsmgpu_adjoint_cfl_dt(self.h, cfl, ctypes.byref(v)), "cfl_dt")
        return v.value

    def set_dt(self, dt):
        gpu.check_rc(gpu.load().lsmgpu_adjoint_set_dt(self.h, float(dt)), "set_dt")

    def set_fields(self, phi0, target, eps):
        self._phi0 = np.array(phi0, dtype=np.float64, order="F", copy=True)
        self._target = np.array(target, dtype=np.float64, order="F", copy=True)
        self._eps = float(eps)
        gpu.check_rc(gpu.load().lsmgpu_adjoint_set_fields(self.h, self._phi0.ctypes.data,
                                                          self._target.ctypes.data,
                                                          float(eps)), "set_fields")

    def forward(self):
        v = ctypes.c_double()
        gpu.check_rc(gpu.load().lsmgpu_adjoint_forward(self.h, ctypes.byref(v)), "forward")
        return v.value

    def backward(self, seed=1.0):
        gt = np.zeros((3, self.lattice, self.lattice, self.lattice))
        gp = np.zeros(self.shape, order="F")
        gpu.check_rc(gpu.load().lsmgpu_adjoint_backward(self.h, float(seed), gt.ctypes.data,
                                                        gp.ctypes.data), "backward")
        return gt, gp

    def timing(self):
        f, a = ctypes.c_float(), ctypes.c_float()
        gpu.check_rc(gpu.load().lsmgpu_adjoint_timing(self.h, ctypes.byref(f),
                                                      ctypes.byref(a)), "timing")
        return f.value, a.value

    def phi_final(self):
        out = np.zeros(self.shape, order="F")
        gpu.check_rc(gpu.load().lsmgpu_adjoint_phi_final(self.h, out.ctypes.data), "phi_final")
        return out


def heaviside(x, eps):
    """LSM_HEAVISIDE (lsm_calculus_toolbox.h:41-45), elementwise."""
    x = np.asarray(x, dtype=np.float64)
    h = 0.5 * (1.0 + x / eps + np.sin(np.pi * x / eps) / np.pi)
    return np.where(x < -eps, 0.0, np.where(x > eps, 1.0, h))


def loss_difference(phi_a, phi_b, target, eps, vol):
    """J(phi_a) - J(phi_b) for two final states (interior arrays), formed
    cell by cell as (Ha - Hb)(Ha + Hb - 2 Ht) so that a finite difference of
    nearby states does not lose its digits to the rounding of two totals."""
    ha, hb, ht = heaviside(phi_a, eps), heaviside(phi_b, eps), heaviside(target, eps)
    return float(np.sum((ha - hb) * (ha + hb - 2.0 * ht)) * vol)


def spline_velocity(theta, n, dx, x_lo, lattice, ghost=3):
    """Host evaluation of the trilinear B-spline velocity on the ghost box
    (the same hat functions as the device kernel); zero in ghost cells."""
    theta = np.asarray(theta, dtype=np.float64).reshape(3, lattice, lattice, lattice)
    vel = [np.zeros(tuple(v + 2 * ghost for v in n), order="F") for _ in range(3)]
    idx, wts = [], []
    for d in range(3):
        h = n[d] * dx[d] / (lattice - 1)
        x = x_lo[d] + (np.arange(n[d]) + 0.5) * dx[d]
        r = (x - x_lo[d]) / h
        a = np.clip(np.floor(r).astype(int), 0, lattice - 2)
        idx.append(a)
        wts.append(r - a)
    for comp in range(3):
        out = np.zeros(n)
        for c in (0, 1):
            for b in (0, 1):
                for a in (0, 1):
                    w = ((wts[0] if a else 1 - wts[0])[:, None, None] *
                         (wts[1] if b else 1 - wts[1])[None, :, None] *
                         (wts[2] if c else 1 - wts[2])[None, None, :])
                    coef = theta[comp][(idx[2] + c)[None, None, :],
                                       (idx[1] + b)[None, :, None],
                                       (idx[0] + a)[:, None, None]]
                    out += w * coef
        vel[comp][ghost:-ghost, ghost:-ghost, ghost:-ghost] = out
    return vel
