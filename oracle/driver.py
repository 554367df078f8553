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
        """A ghost-box Field holding a copy of data (the steppers update their
        Fields in place, so the caller's array is never modified)."""
        return Field(np.array(data, dtype=np.float64, order="F", copy=True), self.gb_lo)

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

    def __init__(self, tb, grid, bc="linear"):
        self.tb, self.g, self.bc = tb, grid, bc
        self.rhs = grid.zeros()
        self.grads = {k: grid.zeros() for k in GRADS_PM}
        self.up = {k: grid.zeros() for k in ("phi_x", "phi_y", "phi_z")}
        self.stage1 = grid.zeros()
        self.stage2 = grid.zeros()

    # -- building blocks ----------------------------------------------------
    def ghost_fill(self, phi):
        """Ghost cells of all six faces in the reference's face order: linear
        extrapolation (LSM3D_LINEAR_EXTRAPOLATION), copy extrapolation
        (LSM3D_COPY_EXTRAPOLATION) or periodic images (the periodic domains
        of the reference's SAMRAI examples, e.g.
        examples/parallel/3d/advection/advection_3d.input:48)."""
        if self.bc == "periodic":
            g = self.g.ghost
            a = phi.data
            for ax in range(3):
                n = self.g.n[ax]
                sl = [slice(None)] * 3
                src = [slice(None)] * 3
                sl[ax], src[ax] = slice(0, g), slice(n, n + g)
                a[tuple(sl)] = a[tuple(src)]
                sl[ax], src[ax] = slice(n + g, n + 2 * g), slice(g, 2 * g)
                a[tuple(sl)] = a[tuple(src)]
            return
        sym = ("lsm3dcopyextrapolation_" if self.bc == "copy"
               else "lsm3dlinearextrapolation_")
        for face in range(6):
            self.tb.call(sym, {"phi": phi}, self.g.fb, bdry_location_idx=face)

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


class PatchedNormalStepper:
    """Normal-velocity steps with reinitialization over z-slab patches run by
    a thread pool -- the reference's own parallel strategy (patch loops over
    the toolbox routines, a 3-cell ghost exchange before every stage and a
    global minimum of dt; LevelSetFunctionIntegrator.cc:382, :567, :1377).
    ctypes releases the GIL during each routine, so patches run in parallel.
    Interior results equal the single-grid Stepper's bit for bit."""

    def __init__(self, tb, grid, nthreads):
        import concurrent.futures
        self.g = grid
        self.nthreads = max(1, int(nthreads))
        nz = grid.n[2]
        npatch = max(1, min(self.nthreads, nz // 4))
        cuts = [grid.fb_lo[2] + (nz * p) // npatch for p in range(npatch + 1)]
        self.patches = []
        for p in range(npatch):
            klo, khi = cuts[p], cuts[p + 1] - 1
            pg = Grid((grid.n[0], grid.n[1], khi - klo + 1), ghost=grid.ghost,
                      lo=(grid.fb_lo[0], grid.fb_lo[1], klo), dx=grid.dx)
            self.patches.append((pg, Stepper(tb, pg)))
        self.pool = concurrent.futures.ThreadPoolExecutor(self.nthreads)

    def scatter(self, full):
        """Per-patch copies of a global Field (interior plus halo)."""
        out = []
        for pg, _ in self.patches:
            f = pg.zeros()
            f.data[...] = full.view(pg.gb_lo, pg.gb_hi)
            out.append(f)
        return out

    def gather(self, parts, full):
        for (pg, _), f in zip(self.patches, parts):
            full.view(pg.fb_lo, pg.fb_hi)[...] = pg.interior(f)

    def exchange(self, parts):
        """z-halo planes from the neighbouring patches' interiors; the global
        z faces get the linear extrapolation."""
        for p, ((pg, st), f) in enumerate(zip(self.patches, parts)):
            if p > 0:
                qg, _ = self.patches[p - 1]
                lo = (pg.gb_lo[0], pg.gb_lo[1], pg.gb_lo[2])
                hi = (pg.gb_hi[0], pg.gb_hi[1], pg.fb_lo[2] - 1)
                f.view(lo, hi)[...] = parts[p - 1].view(lo, hi)
            if p + 1 < len(parts):
                lo = (pg.gb_lo[0], pg.gb_lo[1], pg.fb_hi[2] + 1)
                hi = (pg.gb_hi[0], pg.gb_hi[1], pg.gb_hi[2])
                f.view(lo, hi)[...] = parts[p + 1].view(lo, hi)

    def _fill(self, p, f):
        pg, st = self.patches[p]
        faces = [0, 1, 2, 3]
        if p == 0:
            faces.append(4)
        if p == len(self.patches) - 1:
            faces.append(5)
        for face in faces:
            st.tb.call("lsm3dlinearextrapolation_", {"phi": f}, pg.fb,
                       bdry_location_idx=face)

    def _map(self, fn):
        return list(self.pool.map(fn, range(len(self.patches))))

    def _stage_rhs(self, parts, rhs_kind, aux, phi0s=None, use0=0):
        self.exchange(parts)

        def work(p):
            pg, st = self.patches[p]
            f = parts[p]
            self._fill(p, f)
            if rhs_kind == "normal":
                st.zero_rhs()
                st.weno_pm(f)
                d = dict(st.grads)
                d.update({"lse_rhs": st.rhs, "vel_n": aux[p]})
                st.tb.call("lsm3daddnormalveltermtolserhs_", d, pg.fb)
            else:
                st.weno_pm(f)
                d = dict(st.grads)
                d.update({"reinit_rhs": st.rhs, "phi": f, "phi0": phi0s[p]})
                st.tb.call("lsm3dcomputereinitializationeqnrhs_", d, pg.fb,
                           use_phi0_for_sgn=use0, **pg.dxyz())
        self._map(work)

    def _rk(self, s, outs, uss, ucs, dt):
        self._map(lambda p: self.patches[p][1].rk(s, outs[p], uss[p] if uss else None,
                                                  ucs[p], dt))

    def normal_step(self, parts, Fs, cfl):
        self.exchange(parts)

        def dtp(p):
            pg, st = self.patches[p]
            self._fill(p, parts[p])
            st.weno_pm(parts[p])
            d = dict(st.grads)
            d["vel_n"] = Fs[p]
            return st.tb.call("lsm3dcomputestablenormalveldt_", d, pg.fb,
                              cfl_number=cfl, **pg.dxyz())["dt"]
        dt = min(self._map(dtp))         # minReduction of the patch dts
        s1 = [st.stage1 for _, st in self.patches]
        s2 = [st.stage2 for _, st in self.patches]
        self._stage_rhs(parts, "normal", Fs)
        self._rk(1, s1, None, parts, dt)
        self._stage_rhs(s1, "normal", Fs)
        self._rk(2, s2, s1, parts, dt)
        self._stage_rhs(s2, "normal", Fs)
        self._rk(3, parts, s2, parts, dt)
        return dt

    def reinit(self, parts, cfl, iters, use0=0):
        dtr = cfl * min(self.g.dx)
        phi0s = [f.copy() for f in parts]
        s1 = [st.stage1 for _, st in self.patches]
        s2 = [st.stage2 for _, st in self.patches]
        for _ in range(iters):
            self._stage_rhs(parts, "reinit", None, phi0s, use0)
            self._rk(1, s1, None, parts, dtr)
            self._stage_rhs(s1, "reinit", None, phi0s, use0)
            self._rk(2, s2, s1, parts, dtr)
            self._stage_rhs(s2, "reinit", None, phi0s, use0)
            self._rk(3, parts, s2, parts, dtr)


def deformation_velocity(grid, x_lo, t, period=3.0):
    """LeVeque's 3D deformation field at time t on the ghost box."""
    x, y, z = grid.centers(x_lo)
    g = np.cos(np.pi * t / period)
    u = 2.0 * np.sin(np.pi * x) ** 2 * np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z) * g
    v = -np.sin(2 * np.pi * x) * np.sin(np.pi * y) ** 2 * np.sin(2 * np.pi * z) * g
    w = -np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.sin(np.pi * z) ** 2 * g
    return [grid.field(a) for a in (u, v, w)]
