"""Reference-order time stepping on top of a toolbox (oracle or reference).

TEST INFRASTRUCTURE ONLY.  These loops chain the toolbox routines in the order
of the reference's integrators, one routine call per step of that order:

* TVD-RK3 stage s of the level set equation
  (LevelSetFunctionIntegrator.cc:1319-1510): linear-extrapolation ghost fill
  of the stage input on all six faces (lsm_boundary_conditions.c:227-293,
  case 9) -> LSM3D_ZERO_OUT_LEVEL_SET_EQN_RHS -> LSM3D_UPWIND_HJ_WENO5 +
  LSM3D_ADD_ADVECTION_TERM_TO_LSE_RHS (external velocity) or LSM3D_HJ_WENO5 +
  LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS (normal velocity) -> LSM3D_TVD_RK3_STAGEs;
* the normal-velocity dt (computeStableDt, :345-587): ghost fill ->
  LSM3D_HJ_WENO5 -> LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT;
* reinitialization pseudo-steps (ReinitializationAlgorithm.cc:269-329 with
  dt = cfl*min(dx), :216, sign flag 0 as at :900): ghost fill ->
  LSM3D_HJ_WENO5 -> LSM3D_COMPUTE_REINITIALIZATION_EQN_RHS -> stage.

Arrays are :class:`lsmlib_b200.toolbox.Field` objects on the host.
"""
import numpy as np

from lsmlib_b200.toolbox import Field

GRADS_PM = ("phi_x_plus", "phi_y_plus", "phi_z_plus",
            "phi_x_minus", "phi_y_minus", "phi_z_minus")


class Grid:
    """Ghost box and fill box of a level-set grid (the reference's Grid
    index-space convention, src/serial/lsm_grid.h:43-95)."""

    def __init__(self, n, ghost=3, lo=(0, 0, 0), dx=(1.0, 1.0, 1.0)):
        self.n = tuple(int(v) for v in n)
        self.ghost = int(ghost)
        self.fb_lo = tuple(lo)
        self.fb_hi = tuple(l + m - 1 for l, m in zip(lo, n))
        self.gb_lo = tuple(l - ghost for l in self.fb_lo)
        self.gb_hi = tuple(h + ghost for h in self.fb_hi)
        self.dx = tuple(float(v) for v in dx)

    @property
    def fb(self):
        return (self.fb_lo[0], self.fb_hi[0], self.fb_lo[1], self.fb_hi[1],
                self.fb_lo[2], self.fb_hi[2])

    @property
    def gb(self):
        return (self.gb_lo[0], self.gb_hi[0], self.gb_lo[1], self.gb_hi[1],
                self.gb_lo[2], self.gb_hi[2])

    @property
    def shape(self):
        return tuple(h - l + 1 for l, h in zip(self.gb_lo, self.gb_hi))

    def zeros(self):
        return Field.zeros(self.gb_lo, self.gb_hi)

    def field(self, data):
        return Field(np.asfortranarray(data, dtype=np.float64), self.gb_lo)

    def interior(self, f):
        return f.view(self.fb_lo, self.fb_hi)

    def centers(self, x_lo):
        """Cell-centre coordinates over the ghost box: x_lo + (i + 1/2) dx."""
        ax = [x_lo[d] + (np.arange(self.gb_lo[d], self.gb_hi[d] + 1) + 0.5) * self.dx[d]
              for d in range(3)]
        return np.meshgrid(*ax, indexing="ij")

    def dxyz(self):
        return {"dx": self.dx[0], "dy": self.dx[1], "dz": self.dx[2]}


class Stepper:
    """Reference-order TVD-RK3 loops over one toolbox and one grid."""

    def __init__(self, tb, grid):
        self.tb, self.g = tb, grid
        self.rhs = grid.zeros()
        self.grads = {k: grid.zeros() for k in GRADS_PM}
        self.up = {k: grid.zeros() for k in ("phi_x", "phi_y", "phi_z")}
        self.stage1 = grid.zeros()
        self.stage2 = grid.zeros()

    # -- building blocks ----------------------------------------------------
    def ghost_fill(self, phi):
        for face in range(6):
            self.tb.call("lsm3dlinearextrapolation_", {"phi": phi}, self.g.fb,
                         bdry_location_idx=face)

    def weno_pm(self, phi):
        f = dict(self.grads)
        f["phi"] = phi
        self.tb.call("lsm3dhjweno5_", f, self.g.fb, **self.g.dxyz())

    def rk(self, s, out, us, uc, dt):
        fb = self.g.fb
        if s == 1:
            self.tb.call("lsm3dtvdrk3stage1_", {"u_stage1": out, "u_cur": uc,
                                                "rhs": self.rhs}, fb, dt=dt)
        elif s == 2:
            self.tb.call("lsm3dtvdrk3stage2_", {"u_stage2": out, "u_stage1": us,
                                                "u_cur": uc, "rhs": self.rhs}, fb, dt=dt)
        else:
            self.tb.call("lsm3dtvdrk3stage3_", {"u_next": out, "u_stage2": us,
                                                "u_cur": uc, "rhs": self.rhs}, fb, dt=dt)

    def zero_rhs(self):
        self.tb.call("lsm3dzerooutlevelseteqnrhs_", {"lse_rhs": self.rhs}, self.g.fb)

    def rhs_advect(self, phi, vel):
        self.ghost_fill(phi)
        self.zero_rhs()
        f = dict(self.up)
        f.update({"phi": phi, "vel_x": vel[0], "vel_y": vel[1], "vel_z": vel[2]})
        self.tb.call("lsm3dupwindhjweno5_", f, self.g.fb, **self.g.dxyz())
        self.tb.call("lsm3daddadvectiontermtolserhs_",
                     {"lse_rhs": self.rhs, "phi_x": self.up["phi_x"],
                      "phi_y": self.up["phi_y"], "phi_z": self.up["phi_z"],
                      "vel_x": vel[0], "vel_y": vel[1], "vel_z": vel[2]}, self.g.fb)

    def rhs_normal(self, phi, F):
        self.ghost_fill(phi)
        self.zero_rhs()
        self.weno_pm(phi)
        f = dict(self.grads)
        f.update({"lse_rhs": self.rhs, "vel_n": F})
        self.tb.call("lsm3daddnormalveltermtolserhs_", f, self.g.fb)

    def rhs_reinit(self, phi, phi0, use0):
        self.ghost_fill(phi)
        self.weno_pm(phi)
        f = dict(self.grads)
        f.update({"reinit_rhs": self.rhs, "phi": phi, "phi0": phi0})
        self.tb.call("lsm3dcomputereinitializationeqnrhs_", f, self.g.fb,
                     use_phi0_for_sgn=use0, **self.g.dxyz())

    # -- time steps ---------------------------------------------------------
    def advect_dt(self, vel, cfl):
        r = self.tb.call("lsm3dcomputestableadvectiondt_",
                         {"vel_x": vel[0], "vel_y": vel[1], "vel_z": vel[2]},
                         self.g.fb, cfl_number=cfl, **self.g.dxyz())
        return r["dt"]

    def normal_dt(self, phi, F, cfl):
        self.ghost_fill(phi)
        self.weno_pm(phi)
        f = dict(self.grads)
        f["vel_n"] = F
        return self.tb.call("lsm3dcomputestablenormalveldt_", f, self.g.fb,
                            cfl_number=cfl, **self.g.dxyz())["dt"]

    def advect_step(self, phi, vel_fn, dt):
        """One TVD-RK3 step; vel_fn(c) gives the velocity Fields at t + c*dt."""
        self.rhs_advect(phi, vel_fn(0.0))
        self.rk(1, self.stage1, None, phi, dt)
        self.rhs_advect(self.stage1, vel_fn(1.0))
        self.rk(2, self.stage2, self.stage1, phi, dt)
        self.rhs_advect(self.stage2, vel_fn(0.5))
        self.rk(3, phi, self.stage2, phi, dt)

    def normal_step(self, phi, F, cfl):
        dt = self.normal_dt(phi, F, cfl)
        self.rhs_normal(phi, F)
        self.rk(1, self.stage1, None, phi, dt)
        self.rhs_normal(self.stage1, F)
        self.rk(2, self.stage2, self.stage1, phi, dt)
        self.rhs_normal(self.stage2, F)
        self.rk(3, phi, self.stage2, phi, dt)
        return dt

    def reinit(self, phi, cfl, iters, use0=0):
        dtr = cfl * min(self.g.dx)
        phi0 = phi.copy()
        for _ in range(iters):
            self.rhs_reinit(phi, phi0, use0)
            self.rk(1, self.stage1, None, phi, dtr)
            self.rhs_reinit(self.stage1, phi0, use0)
            self.rk(2, self.stage2, self.stage1, phi, dtr)
            self.rhs_reinit(self.stage2, phi0, use0)
            self.rk(3, phi, self.stage2, phi, dtr)


def deformation_velocity(grid, x_lo, t, period=3.0):
    """LeVeque's 3D deformation field at time t on the ghost box."""
    x, y, z = grid.centers(x_lo)
    g = np.cos(np.pi * t / period)
    u = 2.0 * np.sin(np.pi * x) ** 2 * np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z) * g
    v = -np.sin(2 * np.pi * x) * np.sin(np.pi * y) ** 2 * np.sin(2 * np.pi * z) * g
    w = -np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.sin(np.pi * z) ** 2 * g
    return [grid.field(a) for a in (u, v, w)]
