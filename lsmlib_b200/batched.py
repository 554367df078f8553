"""Python front end of the batched-grid driver (lsmgpu_batch_* of liblsmgpu.so).

``Batch(sizes, dx, precision)`` packs many level-set grids of uneven sizes
into one device buffer; ``set_velocity`` assigns each grid a constant
velocity and its CFL dt; ``advect(nsteps, mode)`` runs TVD-RK3 steps with one
persistent work-list launch per stage (mode 0 replays a CUDA graph).
"""
import ctypes

import numpy as np

from . import gpu
from .ext_abi import dbls, ints

MODE_GRAPH, MODE_PERSISTENT, MODE_PER_GRID = 0, 1, 2
# batch configurations: tile shape c % 5 (32x8x16, 32x8x32, 32x8x64, 16x8x16,
# 16x8x32 cells) with halo-staging schedule c // 5 (0 shared plane, 1 direct
# loads, 2 two cells per thread)
N_CONFIGS = 15
BC_LINEAR, BC_COPY, BC_PERIODIC = 0, 1, 2


class Batch:
    def __init__(self, sizes, dx, precision=8):
        lib = gpu.load()
        self.sizes = [tuple(int(v) for v in s) for s in sizes]
        self.dx = [tuple(float(v) for v in d) for d in dx]
        self.precision = int(precision)
        self.dtype = np.float64 if precision == 8 else np.float32
        flat_n = [v for s in self.sizes for v in s]
        flat_dx = [v for d in self.dx for v in d]
        h = ctypes.c_void_p()
        gpu.check_rc(lib.lsmgpu_batch_create(ctypes.byref(h), len(self.sizes),
                                             ints(flat_n), dbls(flat_dx),
                                             self.precision), "batch_create")
        self.h = h
        self.total = lib.lsmgpu_batch_total_elements(h)
        self.cells = lib.lsmgpu_batch_cells(h)
        self.offsets = []
        for g in range(len(self.sizes)):
            off = ctypes.c_longlong()
            gb = (ctypes.c_int * 6)()
            gpu.check_rc(lib.lsmgpu_batch_grid(h, g, ctypes.byref(off), gb), "batch_grid")
            self.offsets.append(off.value)

    def close(self):
        if self.h:
            gpu.load().lsmgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, g):
        return tuple(n + 6 for n in self.sizes[g])

    def pack(self, fields):
        """Host packed buffer from per-grid Fortran-ordered ghost-box arrays."""
        buf = np.zeros(self.total, dtype=self.dtype)
        for g, f in enumerate(fields):
            a = np.asarray(f, dtype=self.dtype)
            buf[self.offsets[g]:self.offsets[g] + a.size] = a.ravel(order="F")
        return buf

    def unpack(self, buf):
        out = []
        for g in range(len(self.sizes)):
            shp = self.shape(g)
            n = int(np.prod(shp))
            out.append(buf[self.offsets[g]:self.offsets[g] + n].reshape(shp, order="F"))
        return out

    def upload(self, fields):
        buf = self.pack(fields)
        gpu.check_rc(gpu.load().lsmgpu_batch_upload(self.h, buf.ctypes.data), "batch_upload")

    def download(self):
        buf = np.empty(self.total, dtype=self.dtype)
        gpu.check_rc(gpu.load().lsmgpu_batch_download(self.h, buf.ctypes.data),
                     "batch_download")
        return self.unpack(buf)

    def set_velocity(self, vel, cfl=0.5):
        flat = [v for u in vel for v in u]
        gpu.check_rc(gpu.load().lsmgpu_batch_set_velocity(self.h, dbls(flat), cfl),
                     "batch_set_velocity")

    def dt(self):
        out = (ctypes.c_double * len(self.sizes))()
        gpu.check_rc(gpu.load().lsmgpu_batch_get_dt(self.h, out), "batch_get_dt")
        return list(out)

    def set_tile(self, shape):
        gpu.check_rc(gpu.load().lsmgpu_batch_set_tile(self.h, int(shape)), "batch_set_tile")

    def tile(self):
        s = ctypes.c_int()
        t = (ctypes.c_int * 3)()
        gpu.check_rc(gpu.load().lsmgpu_batch_get_tile(self.h, ctypes.byref(s), t),
                     "batch_get_tile")
        return s.value, tuple(t)

    def set_bc(self, kind):
        gpu.check_rc(gpu.load().lsmgpu_batch_set_bc(self.h, int(kind)), "batch_set_bc")

    def set_fp64_policy(self, policy):
        """FP32 batches: integrator.FP64_KINKS | integrator.STOCH_ROUND."""
        gpu.check_rc(gpu.load().lsmgpu_batch_set_fp64_policy(self.h, int(policy)),
                     "batch_set_fp64_policy")

    def set_fp64_kinks(self, on):
        gpu.check_rc(gpu.load().lsmgpu_batch_set_fp64_kinks(self.h, int(on)),
                     "batch_set_fp64_kinks")

    def autotune(self, report=True):
        """Times the N_CONFIGS configurations (5 tile shapes x 3 halo-staging
        schedules) and keeps the fastest; returns their ms per step."""
        ms = (ctypes.c_float * N_CONFIGS)() if report else None
        gpu.check_rc(gpu.load().lsmgpu_batch_autotune(self.h, ms), "batch_autotune")
        return list(ms) if report else None

    def advect(self, nsteps, mode=MODE_GRAPH, sync=True):
        gpu.check_rc(gpu.load().lsmgpu_batch_advect_tvdrk3(self.h, int(nsteps), int(mode),
                                                           int(sync)), "batch_advect")

    def stream(self):
        return gpu.load().lsmgpu_batch_stream(self.h)
