"""Level-set grids and time stepping on torch tensors (the host driver).

``Grid`` mirrors the serial package's grid (src/serial/lsm_grid.h:43-95,
lsm_grid.c:50-210, :788-982): the interior spans [x_lo, x_hi] with grid_dims
cells of spacing dx, every field carries a ghost layer whose width depends on
the spatial accuracy ({LOW: 2, MEDIUM: 3, HIGH: 5, VERY_HIGH: 4},
lsm_grid.c:46), index spaces start at 0 on the ghost box, grid point i sits
at x_lo_ghostbox + i dx (lsm_initialization3d.c:55-57), and the fill box of
the derivative schemes is the reference's (setIndexSpaceLimits*).

``LevelSetIntegrator`` advances such fields with the fused TVD-RK3 drivers of
liblsmgpu.so: normal speed with periodic reinitialization, external velocity,
the deformation field, and reinitialization alone.  Fields are CUDA tensors
of shape grid.shape = grid_dims_ghostbox reversed (z, y, x), so that x is the
fastest index as in the reference's Fortran arrays.  The work is enqueued on
torch's current CUDA stream.
"""
import math

import numpy as np
import torch

from lsmlib_b200 import gpu, integrator

ACCURACY_GHOSTCELLS = {"LOW": 2, "MEDIUM": 3, "HIGH": 5, "VERY_HIGH": 4}
SCHEME_WIDTH = {"LOW": 1, "MEDIUM": 2, "HIGH": 3, "VERY_HIGH": 3}
BOUNDARIES = {"linear": integrator.BC_LINEAR, "copy": integrator.BC_COPY,
              "periodic": integrator.BC_PERIODIC}


class Grid:
    """A 3D level-set grid (the reference's Grid structure)."""

    def __init__(self, grid_dims, x_lo, x_hi, dx, accuracy="VERY_HIGH"):
        if accuracy not in ACCURACY_GHOSTCELLS:
            raise ValueError("accuracy is one of %s" % sorted(ACCURACY_GHOSTCELLS))
        g = ACCURACY_GHOSTCELLS[accuracy]
        self.num_dims = 3
        self.accuracy = accuracy
        self.num_ghostcells = g
        self.grid_dims = tuple(int(v) for v in grid_dims)
        self.dx = tuple(float(v) for v in dx)
        self.x_lo = tuple(float(v) for v in x_lo)
        self.x_hi = tuple(float(v) for v in x_hi)
        self.grid_dims_ghostbox = tuple(n + 2 * g for n in self.grid_dims)
        self.x_lo_ghostbox = tuple(lo - g * h for lo, h in zip(self.x_lo, self.dx))
        self.x_hi_ghostbox = tuple(hi + g * h for hi, h in zip(self.x_hi, self.dx))
        self.num_gridpts = math.prod(self.grid_dims_ghostbox)
        # index spaces (setIndexSpaceLimitsCentral and the scheme's limits)
        gd = self.grid_dims_ghostbox
        self.gb = (0, gd[0] - 1, 0, gd[1] - 1, 0, gd[2] - 1)
        self.D1_fb = (1, gd[0] - 2, 1, gd[1] - 2, 1, gd[2] - 2)
        self.D2_fb = (2, gd[0] - 3, 2, gd[1] - 3, 2, gd[2] - 3)
        self.D3_fb = (3, gd[0] - 4, 3, gd[1] - 4, 3, gd[2] - 4)
        # setIndexSpaceLimitsENO1/ENO2/ENO3/WENO5 (lsm_grid.c:831-982): the
        # scheme's fill box is the D1 box shrunk by these amounts (D2 and D3
        # boxes are the ghost box shrunk by 2 and 3)
        lo_shift, hi_shift = {"LOW": (0, 1), "MEDIUM": (2, 2), "HIGH": (3, 4),
                              "VERY_HIGH": (2, 3)}[accuracy]
        d = self.D1_fb
        self.fb = (d[0] + lo_shift, d[1] - hi_shift, d[2] + lo_shift, d[3] - hi_shift,
                   d[4] + lo_shift, d[5] - hi_shift)
        (self.ilo_gb, self.ihi_gb, self.jlo_gb, self.jhi_gb, self.klo_gb,
         self.khi_gb) = self.gb
        (self.ilo_fb, self.ihi_fb, self.jlo_fb, self.jhi_fb, self.klo_fb,
         self.khi_fb) = self.fb
        # narrow-band parameters of the serial package's local method, as
        # setIndexSpaceLimits sets them (lsm_grid.c:986-1005); carried into
        # grid files
        self.num_nb_levels = g
        self.mark_gb, self.mark_D1, self.mark_D2, self.mark_D3 = 120, 119, 118, 117
        self.mark_fb = 120 - g
        wide = accuracy in ("HIGH", "VERY_HIGH")
        self.beta = (3 if wide else 2) * self.dx[0]
        self.gamma = (6 if wide else 4) * self.dx[0]

    # -- constructors of lsm_grid.c -------------------------------------------
    @classmethod
    def set_dx(cls, dx, x_lo, x_hi, accuracy="VERY_HIGH"):
        """createGridSetDx / createGridSetDxDyDz (lsm_grid.c:50-190): grid_dims
        = rint((x_hi - x_lo) / dx), x_hi reset to x_lo + grid_dims dx."""
        dx = (float(dx),) * 3 if not hasattr(dx, "__len__") else tuple(map(float, dx))
        dims = [int(round((h - l) / d)) for l, h, d in zip(x_lo, x_hi, dx)]
        hi = [l + n * d for l, n, d in zip(x_lo, dims, dx)]
        return cls(dims, x_lo, hi, dx, accuracy)

    @classmethod
    def set_grid_dims(cls, grid_dims, x_lo, x_hi, accuracy="VERY_HIGH"):
        """createGridSetGridDims (lsm_grid.c:196-250): dx = (x_hi - x_lo) /
        grid_dims."""
        dx = [(h - l) / n for l, h, n in zip(x_lo, x_hi, grid_dims)]
        return cls(grid_dims, x_lo, x_hi, dx, accuracy)

    # -- grid files (lsm_grid.c:613-787) -------------------------------------------
    def write_binary(self, file_name, zip_status=0):
        """writeGridToBinaryFile: the fields in the reference's order, native
        ints and doubles with no padding; zip_status 1 (GZIP) or 2 (BZIP2)
        compresses the file to name.gz / name.bz2.  Returns the name
        written."""
        from .data_arrays import _write
        ints = lambda v: np.asarray(v, dtype=np.intc).tobytes()
        reals = lambda v: np.asarray(v, dtype=np.float64).tobytes()
        payload = b"".join([
            ints([self.num_dims]), reals(self.x_lo), reals(self.x_hi),
            reals(self.x_lo_ghostbox), reals(self.x_hi_ghostbox), ints(self.grid_dims),
            ints(self.grid_dims_ghostbox), reals(self.dx), ints([self.num_gridpts]),
            ints(self.gb), ints(self.fb), ints(self.D1_fb), ints(self.D2_fb),
            ints(self.D3_fb), ints([self.num_nb_levels]),
            bytes([self.mark_gb, self.mark_D1, self.mark_D2, self.mark_D3, self.mark_fb]),
            reals([self.beta]), reals([self.gamma])])
        return _write(file_name, payload, zip_status)

    def describe(self):
        """printGrid (lsm_grid.c:322-440): the grid as the reference prints it,
        3D form (C's %g for reals, %u for the marks)."""
        r = lambda v: "%g" % v

        def box(b):
            return "[%d,%d] x [%d,%d] x [%d,%d]" % tuple(b)
        lines = [
            "Number of dimensions: %d" % self.num_dims,
            "Geometric limits (without ghostcells): [%s,%s] x [%s,%s] x [%s,%s]" % tuple(
                r(v) for pair in zip(self.x_lo, self.x_hi) for v in pair),
            "Geometric limits (with ghostcells): [%s,%s] x [%s,%s] x [%s,%s]" % tuple(
                r(v) for pair in zip(self.x_lo_ghostbox, self.x_hi_ghostbox) for v in pair),
            "Grid size (without ghostcells): %d x %d x %d" % tuple(self.grid_dims),
            "Grid size (with ghostcells): %d x %d x %d" % tuple(self.grid_dims_ghostbox),
            "Grid spacing: dx = %s, dy = %s, dz = %s " % tuple(r(v) for v in self.dx),
            "Total number of grid points: %d" % self.num_gridpts,
            "Ghost box index limits: " + box(self.gb),
            "Fill box index limits: " + box(self.fb),
            "1st order differences fill box: " + box(self.D1_fb),
            "2nd order differences fill box: " + box(self.D2_fb),
            "3rd order differences fill box: " + box(self.D3_fb),
            "Number of narrow band levels (local method) %d" % self.num_nb_levels,
            "Boundary layer marks (local method) gb %u D1 %u D2 %u D3 %u fb %u" % (
                self.mark_gb, self.mark_D1, self.mark_D2, self.mark_D3, self.mark_fb),
            "Narrow band width (local method) beta(inner) %s gamma(outer) %s" % (
                r(self.beta), r(self.gamma)),
        ]
        return "\n".join(lines) + "\n"

    def write_ascii(self, file_name, zip_status=0):
        """writeGridToAsciiFile (lsm_grid.c:601-611): the printGrid text,
        optionally compressed to name.gz / name.bz2.  Returns the name
        written."""
        from .data_arrays import _write
        return _write(file_name, self.describe().encode(), zip_status)

    @classmethod
    def read_binary(cls, file_name):
        """readGridFromBinaryFile: every field as the file holds it (names
        ending in .gz / .bz2 are decompressed).  The accuracy is the one
        whose ghost width the file's narrow-band level count gives."""
        from .data_arrays import _read
        raw = _read(file_name)
        pos = 0

        def take(dtype, n):
            nonlocal pos
            size = np.dtype(dtype).itemsize * n
            if pos + size > len(raw):
                raise ValueError("%s: truncated grid file" % file_name)
            v = np.frombuffer(raw[pos:pos + size], dtype=dtype)
            pos += size
            return v

        g = cls.__new__(cls)
        g.num_dims = int(take(np.intc, 1)[0])
        for name in ("x_lo", "x_hi", "x_lo_ghostbox", "x_hi_ghostbox"):
            setattr(g, name, tuple(float(v) for v in take(np.float64, 3)))
        g.grid_dims = tuple(int(v) for v in take(np.intc, 3))
        g.grid_dims_ghostbox = tuple(int(v) for v in take(np.intc, 3))
        g.dx = tuple(float(v) for v in take(np.float64, 3))
        g.num_gridpts = int(take(np.intc, 1)[0])
        for name in ("gb", "fb", "D1_fb", "D2_fb", "D3_fb"):
            setattr(g, name, tuple(int(v) for v in take(np.intc, 6)))
        g.num_nb_levels = int(take(np.intc, 1)[0])
        (g.mark_gb, g.mark_D1, g.mark_D2, g.mark_D3,
         g.mark_fb) = (int(v) for v in take(np.uint8, 5))
        g.beta = float(take(np.float64, 1)[0])
        g.gamma = float(take(np.float64, 1)[0])
        by_width = {w: a for a, w in ACCURACY_GHOSTCELLS.items()}
        g.accuracy = by_width.get(g.num_nb_levels)
        g.num_ghostcells = g.num_nb_levels
        (g.ilo_gb, g.ihi_gb, g.jlo_gb, g.jhi_gb, g.klo_gb, g.khi_gb) = g.gb
        (g.ilo_fb, g.ihi_fb, g.jlo_fb, g.jhi_fb, g.klo_fb, g.khi_fb) = g.fb
        return g

    # -- fields -------------------------------------------------------------------
    @property
    def shape(self):
        """Tensor shape of a field: (nz, ny, nx) of the ghost box."""
        return tuple(reversed(self.grid_dims_ghostbox))

    def coordinates(self, device="cuda", dtype=torch.float64):
        """x, y, z of every grid point, each of shape ``shape``."""
        ax = [self.x_lo_ghostbox[d] + self.dx[d] *
              torch.arange(self.grid_dims_ghostbox[d], dtype=torch.float64)
              for d in range(3)]
        z, y, x = torch.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
        return tuple(t.to(device=device, dtype=dtype).contiguous() for t in (x, y, z))

    def zeros(self, device="cuda", dtype=torch.float64):
        return torch.zeros(self.shape, device=device, dtype=dtype)

    def __repr__(self):
        return ("Grid(grid_dims=%s, x_lo=%s, x_hi=%s, dx=%s, accuracy=%s, fb=%s)"
                % (self.grid_dims, self.x_lo, self.x_hi, self.dx, self.accuracy, self.fb))


class LevelSetIntegrator:
    """TVD-RK3 time stepping of level-set fields on ``grid`` (WENO5 spatial
    derivatives, the reference integrator's call order,
    LevelSetFunctionIntegrator.cc:1319-1510).

    ``fp32_policy`` (torch.float32 only) picks the FP64 parts of the FP32
    form from lsmlib_b200.integrator's FP64_KINKS, FP64_SIGN, STOCH_ROUND
    and FP64_BAND (the tiles within 16 cells of the interface in FP64, for
    ``advance_deformation``)."""

    def __init__(self, grid, dtype=torch.float64, boundary="linear", cfl=0.5,
                 reinit_interval=10, reinit_iters=20, use_phi0_for_sgn=False,
                 fp_mode="fast", fp32_policy=None):
        if grid.num_ghostcells < 3:
            raise ValueError("WENO5 needs 3 ghost cells; use accuracy HIGH or VERY_HIGH")
        if dtype not in (torch.float64, torch.float32):
            raise ValueError("dtype is torch.float64 or torch.float32")
        if boundary not in BOUNDARIES:
            raise ValueError("boundary is one of %s" % sorted(BOUNDARIES))
        self.grid, self.dtype, self.cfl = grid, dtype, float(cfl)
        self.reinit_interval, self.reinit_iters = int(reinit_interval), int(reinit_iters)
        self.use_phi0 = 1 if use_phi0_for_sgn else 0
        self.fp_mode = integrator.FP_FAST if fp_mode == "fast" else integrator.FP_STRICT
        self.steps = 0
        prec = 8 if dtype == torch.float64 else 4
        self._ws = integrator.Workspace(grid.gb, prec)
        self._ws.set_bc(BOUNDARIES[boundary])
        if prec == 4 and fp32_policy is not None:
            self._ws.set_fp64_policy(fp32_policy)

    # -- plumbing -----------------------------------------------------------------
    def _ptr(self, t, what):
        if not (t.is_cuda and t.dtype == self.dtype and t.is_contiguous()
                and tuple(t.shape) == self.grid.shape):
            raise ValueError("%s must be a contiguous CUDA %s tensor of shape %s"
                             % (what, self.dtype, self.grid.shape))
        return _Ptr(t.data_ptr())

    def _enter(self):
        lib = gpu.load()
        gpu.check_rc(lib.lsmgpu_set_stream(torch.cuda.current_stream().cuda_stream),
                     "set_stream")
        self._prev_mode = integrator.get_fp_mode()
        integrator.set_fp_mode(self.fp_mode)

    def _leave(self):
        integrator.set_fp_mode(self._prev_mode)

    # -- drivers ------------------------------------------------------------------
    def advance_normal(self, phi, speed, nsteps=1):
        """phi_t + F |grad phi| = 0 for nsteps CFL steps, reinitializing after
        every reinit_interval-th step (counted over the integrator's life)."""
        p, f = self._ptr(phi, "phi"), self._ptr(speed, "speed")
        self._enter()
        try:
            self._ws.normal(p, f, self.grid.fb, self.grid.dx, cfl=self.cfl, nsteps=nsteps,
                            step0=self.steps, reinit_interval=self.reinit_interval,
                            reinit_iters=self.reinit_iters, use_phi0=self.use_phi0)
        finally:
            self._leave()
        self.steps += int(nsteps)

    def advance_external(self, phi, velocity, nsteps=1, dt=None):
        """phi_t + V.grad phi = 0 with velocity = (u, v, w) tensors, CFL dt
        every step unless ``dt`` is given."""
        p = self._ptr(phi, "phi")
        vel = [self._ptr(v, "velocity") for v in velocity]
        self._enter()
        try:
            self._ws.advect(p, vel, self.grid.fb, self.grid.dx, cfl=self.cfl,
                            dt_fixed=float(dt or 0.0), nsteps=nsteps)
        finally:
            self._leave()
        self.steps += int(nsteps)

    def advance_deformation(self, phi, period, t_end, nsteps=1):
        """LeVeque's deformation field of the given period, dt clipped at t_end;
        the field is evaluated at grid points x_lo_ghostbox + i dx."""
        p = self._ptr(phi, "phi")
        g = self.grid
        # the driver places cell i of the fill box at x_lo + (i + 1/2) dx, so the
        # grid point of index i (x_lo_ghostbox + i dx) needs x_lo shifted by dx/2
        x_lo = tuple(g.x_lo_ghostbox[d] - 0.5 * g.dx[d] for d in range(3))
        self._enter()
        try:
            self._ws.deformation(p, g.fb, g.dx, x_lo, period=period, cfl=self.cfl,
                                 t_end=t_end, nsteps=nsteps)
        finally:
            self._leave()
        self.steps += int(nsteps)

    def reinitialize(self, phi, iters=None):
        """iters TVD-RK3 pseudo-steps of the reinitialization equation with
        dt = cfl min(dx) (ReinitializationAlgorithm.cc:216)."""
        p = self._ptr(phi, "phi")
        self._enter()
        try:
            self._ws.reinit(p, self.grid.fb, self.grid.dx, cfl=self.cfl,
                            iters=int(iters or self.reinit_iters), use_phi0=self.use_phi0)
        finally:
            self._leave()

    @property
    def time(self):
        """Simulated time and the dt of the last step (waits for the stream)."""
        return self._ws.time()

    def close(self):
        self._ws.close()


class _Ptr:
    """A raw device pointer in the form the Workspace calls expect."""

    def __init__(self, p):
        self.ptr = p
