// stage.cuh -- fused TVD Runge-Kutta stage kernels (the performance path).
//
// One kernel evaluates, for every fill-box cell, the HJ-WENO5 derivatives of
// the stage input phi_s, the level-set / reinitialization right-hand side and
// the Runge-Kutta combination, and writes the stage output -- the work of the
// reference's per-stage sequence
//   ghost fill -> LSM3D_ZERO_OUT_LEVEL_SET_EQN_RHS -> LSM3D_(UPWIND_)HJ_WENO5
//   -> LSM3D_ADD_*_TERM_TO_LSE_RHS (or LSM3D_COMPUTE_REINITIALIZATION_EQN_RHS)
//   -> LSM3D_TVD_RK3_STAGE*
// (LevelSetFunctionIntegrator.cc:1319-1510, ReinitializationAlgorithm.cc:
// 269-329) in one pass over HBM.
//
// Data movement (2.5-D marching): a block owns a TX x TY column of cells and
// walks it along z.  Each thread keeps phi(i,j,k-3..k+3) in registers; the
// x/y neighbours of the current plane come from a shared-memory tile with a
// 3-cell halo (only the four side strips; axis-aligned stencils never read
// the corners).  Linear-extrapolation ghost cells
// (lsm_boundary_conditions3d.f:46-170) are produced on the fly: a stencil
// point that leaves the domain box along one axis is
//   phi(edge) + (phi(edge) - phi(edge+-1)) * distance,
// which is exactly the value the reference's face-by-face fill leaves in a
// face ghost cell (corner and edge ghosts are never read by the stencils).
#pragma once
#include "common.cuh"
#include "stencil.cuh"
#include "weno_fast.cuh"

namespace lsmgpu {

enum StageKind {
  kStageAdvect = 0,    // external velocity arrays: upwind WENO5, -V.grad(phi)
  kStageNormal = 1,    // normal speed array: WENO5 +-, Godunov, -F|grad phi|
  kStageReinit = 2,    // reinitialization RHS, sign from phi_s (or phi0)
  kStageNormalRhs = 3  // normal speed, writes L(phi) and CFL maxima only
};

template <typename T>
struct StageParams {
  T* out;              // stage output (fill box written)
  const T* phi_s;      // stage input (stencil read)
  const T* phi_n;      // u_cur of the RK combination
  const T* aux0;       // vel_x | F | phi0
  const T* aux1;       // vel_y
  const T* aux2;       // vel_z
  T* rhs_out;          // kStageNormalRhs: L(phi_s)
  double* partials;    // kStageNormalRhs: per-block CFL maxima
  Box gb;              // ghost box shared by every array
  FillBox fb;          // cells to update
  FillBox dom;         // domain box for on-the-fly ghost extrapolation
  unsigned bc_mask;    // bit f set: extrapolate beyond face f (0..5)
  T inv[3];            // 1/dx, 1/dy, 1/dz
  T dx_sq;             // max(dx,dy,dz)^2 (reinit sign, CFL)
  const double* dt_dev;
  double dt;
  int rk_kind;         // 1, 22, 32, 33 (see rk_update)
  int use_phi0;
  int fp64_kinks;      // FP32 form: recompute kink stencils in FP64
};

template <typename T>
__device__ __forceinline__ T rk_combine(int kind, T uc, T us, T r, T dt) {
  switch (kind) {
    case 22: return T(0.5) * (uc + us + dt * r);
    case 32: return T(0.75) * uc + T(0.25) * (us + dt * r);
    case 33: return (T(1) / T(3)) * uc + (T(2) / T(3)) * (us + dt * r);
    default: return us + dt * r;
  }
}

// phi at (i,j,k) where at most one coordinate may lie outside the domain box
template <typename T>
__device__ __forceinline__ T fetch_bc(const Grid3<const T>& g,
                                      const StageParams<T>& p, int i, int j,
                                      int k) {
  int c[3] = {i, j, k};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (c[d] < p.dom.lo[d] && (p.bc_mask & (1u << (2 * d)))) {
      const int dist = p.dom.lo[d] - c[d];
      c[d] = p.dom.lo[d];
      const T* e = g.ptr(c[0], c[1], c[2]);
      const T e0 = __ldg(e), e1 = __ldg(e + g.stride(d));
      const T slope = e0 - e1;
      return e0 + slope * (T)dist;
    }
    if (c[d] > p.dom.hi[d] && (p.bc_mask & (2u << (2 * d)))) {
      const int dist = c[d] - p.dom.hi[d];
      c[d] = p.dom.hi[d];
      const T* e = g.ptr(c[0], c[1], c[2]);
      const T e0 = __ldg(e), e1 = __ldg(e - g.stride(d));
      const T slope = e0 - e1;
      return e0 + slope * (T)dist;
    }
  }
  return __ldg(g.ptr(i, j, k));
}

// One-sided WENO5 from seven consecutive phi values w[0..6] = phi(c-3..c+3).
template <typename T, bool FAST>
__device__ __forceinline__ T weno_minus7(const T* w, T inv) {
  const T v1 = (w[1] - w[0]) * inv, v2 = (w[2] - w[1]) * inv,
          v3 = (w[3] - w[2]) * inv, v4 = (w[4] - w[3]) * inv,
          v5 = (w[5] - w[4]) * inv;
  return FAST ? weno5_fast(v1, v2, v3, v4, v5) : weno5_strict(v1, v2, v3, v4, v5);
}
template <typename T, bool FAST>
__device__ __forceinline__ T weno_plus7(const T* w, T inv) {
  const T v1 = (w[6] - w[5]) * inv, v2 = (w[5] - w[4]) * inv,
          v3 = (w[4] - w[3]) * inv, v4 = (w[3] - w[2]) * inv,
          v5 = (w[2] - w[1]) * inv;
  return FAST ? weno5_fast(v1, v2, v3, v4, v5) : weno5_strict(v1, v2, v3, v4, v5);
}

// FP32 form: the same values, with kink stencils recomputed in FP64 from the
// FP32 phi values.
template <typename T, bool FAST>
__device__ __forceinline__ T weno_side(const T* w, T inv, bool plus,
                                       bool fp64_kinks) {
  if (sizeof(T) == 4 && fp64_kinks) {
    const T v1 = plus ? (w[6] - w[5]) * inv : (w[1] - w[0]) * inv;
    const T v2 = plus ? (w[5] - w[4]) * inv : (w[2] - w[1]) * inv;
    const T v3 = plus ? (w[4] - w[3]) * inv : (w[3] - w[2]) * inv;
    const T v4 = plus ? (w[3] - w[2]) * inv : (w[4] - w[3]) * inv;
    const T v5 = plus ? (w[2] - w[1]) * inv : (w[5] - w[4]) * inv;
    if (weno5_is_kink(v1, v2, v3, v4, v5)) {
      double wd[7];
#pragma unroll
      for (int m = 0; m < 7; m++) wd[m] = (double)w[m];
      const double id = (double)inv;
      return (T)(plus ? weno_plus7<double, true>(wd, id)
                      : weno_minus7<double, true>(wd, id));
    }
    return weno5_fast(v1, v2, v3, v4, v5);
  }
  return plus ? weno_plus7<T, FAST>(w, inv) : weno_minus7<T, FAST>(w, inv);
}

template <typename T>
__device__ __forceinline__ T godunov_sq2(T vn, T xp, T yp, T zp, T xm, T ym,
                                         T zm) {
  T a, b, s;
  const T z = T(0);
  if (vn > z) {
    a = fmax2(xm, z); b = fmin2(xp, z); s = fmax2(a * a, b * b);
    a = fmax2(ym, z); b = fmin2(yp, z); s = s + fmax2(a * a, b * b);
    a = fmax2(zm, z); b = fmin2(zp, z); s = s + fmax2(a * a, b * b);
  } else {
    a = fmin2(xm, z); b = fmax2(xp, z); s = fmax2(a * a, b * b);
    a = fmin2(ym, z); b = fmax2(yp, z); s = s + fmax2(a * a, b * b);
    a = fmin2(zm, z); b = fmax2(zp, z); s = s + fmax2(a * a, b * b);
  }
  return s;
}

// reinitialization RHS of one cell (lsm_reinitialization3d.f.in:158-199,
// :218-256); the FP32 form evaluates the smoothed sign in FP64
template <typename T>
__device__ __forceinline__ T reinit_cell(T pc, T xp, T yp, T zp, T xm, T ym,
                                         T zm, T dx_sq, bool use0) {
  const T z = T(0);
  T gp[3] = {xp, yp, zp}, gm[3] = {xm, ym, zm}, gs[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (pc > z) {
      gp[d] = fmax2(-gp[d], z);
      gm[d] = fmax2(gm[d], z);
    } else {
      gp[d] = fmax2(gp[d], z);
      gm[d] = fmax2(-gm[d], z);
    }
    gs[d] = fmax2(gp[d], gm[d]);
  }
  if (!(fabsT(pc) >= Consts<T>::zero_tol)) return z;
  const T nsq = gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2];
  if (sizeof(T) == 4) {
    const double pd = pc, nd = nsq, dd = dx_sq;
    const double sgn = use0 ? pd / sqrt(pd * pd + dd) : pd / sqrt(pd * pd + nd * dd);
    return (T)(sgn * (1.0 - sqrt(nd)));
  }
  const T sgn = use0 ? pc / sqrtT(pc * pc + dx_sq)
                     : pc / sqrtT(pc * pc + nsq * dx_sq);
  return sgn * (T(1) - sqrtT(nsq));
}

template <typename T, int KIND, bool FAST, int TX, int TY, int TZ>
__global__ void __launch_bounds__(TX * TY)
k_stage(StageParams<T> p) {
  __shared__ T tile[TY + 6][TX + 6];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = p.fb.lo[0] + (int)blockIdx.x * TX + tx;
  const int j = p.fb.lo[1] + (int)blockIdx.y * TY + ty;
  const int kb = p.fb.lo[2] + (int)blockIdx.z * TZ;
  const int ke = min(kb + TZ - 1, p.fb.hi[2]);
  const bool act = (i <= p.fb.hi[0]) && (j <= p.fb.hi[1]);
  const Grid3<const T> phi = make_grid(p.phi_s, p.gb);
  const long sy = p.gb.sy(), sz = p.gb.sz();
  const long base0 = -((long)p.gb.lo[0] + sy * p.gb.lo[1] + sz * p.gb.lo[2]);
  const T dt = p.dt_dev ? (T)(*p.dt_dev) : (T)p.dt;
  const bool need_bc = p.bc_mask != 0u;
  double hmax = -1.0;

  // Tile roles.  Active threads put their own phi(i,j,k) in the tile.  In a
  // partial tile the cells just past the fill box (up to 3) are halo for the
  // active cells, so inactive threads within 3 cells of it load theirs.  The
  // side strips beyond the tile are loaded by the first/last three threads of
  // each row/column when the cell they serve is active.
  const int hi0 = p.fb.hi[0], hi1 = p.fb.hi[1];
  const bool ctr_halo = !act && i <= hi0 + 3 && j <= hi1 + 3 && !(i > hi0 && j > hi1);
  const int hx = (tx < 3) ? (i - 3) : (i + 3);
  const bool has_hx = (j <= hi1) && ((tx < 3) || (tx >= TX - 3 && i <= hi0));
  const int hj = (ty < 3) ? (j - 3) : (j + 3);
  const bool has_hy = (i <= hi0) && ((ty < 3) || (ty >= TY - 3 && j <= hi1));

  T w[7];
  if (act) {
#pragma unroll
    for (int m = 0; m < 6; m++)
      w[m + 1] = need_bc ? fetch_bc(phi, p, i, j, kb - 3 + m)
                         : __ldg(phi.ptr(i, j, kb - 3 + m));
  }
  for (int k = kb; k <= ke; ++k) {
    if (act) {
#pragma unroll
      for (int m = 0; m < 6; m++) w[m] = w[m + 1];
      w[6] = need_bc ? fetch_bc(phi, p, i, j, k + 3) : __ldg(phi.ptr(i, j, k + 3));
      tile[ty + 3][tx + 3] = w[3];
    } else if (ctr_halo) {
      tile[ty + 3][tx + 3] = need_bc ? fetch_bc(phi, p, i, j, k)
                                     : __ldg(phi.ptr(i, j, k));
    }
    if (has_hx) {
      const int tcol = (tx < 3) ? tx : tx + 6;
      tile[ty + 3][tcol] = need_bc ? fetch_bc(phi, p, hx, j, k)
                                   : __ldg(phi.ptr(hx, j, k));
    }
    if (has_hy) {
      const int trow = (ty < 3) ? ty : ty + 6;
      tile[trow][tx + 3] = need_bc ? fetch_bc(phi, p, i, hj, k)
                                   : __ldg(phi.ptr(i, hj, k));
    }
    __syncthreads();
    if (act) {
      T wx[7], wy[7];
#pragma unroll
      for (int m = 0; m < 7; m++) {
        wx[m] = tile[ty + 3][tx + m];
        wy[m] = tile[ty + m][tx + 3];
      }
      const long o = base0 + (long)i + sy * j + sz * k;
      T L;
      if (KIND == kStageAdvect) {
        // LSM3D_UPWIND_HJ_WENO5 + LSM3D_ADD_ADVECTION_TERM_TO_LSE_RHS
        const T u = __ldg(p.aux0 + o), v = __ldg(p.aux1 + o), ww = __ldg(p.aux2 + o);
        T gx = T(0), gy = T(0), gz = T(0);
        if (!(fabsT(u) < Consts<T>::zero_tol))
          gx = weno_side<T, FAST>(wx, p.inv[0], !(u > T(0)), p.fp64_kinks);
        if (!(fabsT(v) < Consts<T>::zero_tol))
          gy = weno_side<T, FAST>(wy, p.inv[1], !(v > T(0)), p.fp64_kinks);
        if (!(fabsT(ww) < Consts<T>::zero_tol))
          gz = weno_side<T, FAST>(w, p.inv[2], !(ww > T(0)), p.fp64_kinks);
        L = T(0) - (u * gx + v * gy + ww * gz);
      } else {
        const T xp = weno_side<T, FAST>(wx, p.inv[0], true, p.fp64_kinks);
        const T xm = weno_side<T, FAST>(wx, p.inv[0], false, p.fp64_kinks);
        const T yp = weno_side<T, FAST>(wy, p.inv[1], true, p.fp64_kinks);
        const T ym = weno_side<T, FAST>(wy, p.inv[1], false, p.fp64_kinks);
        const T zp = weno_side<T, FAST>(w, p.inv[2], true, p.fp64_kinks);
        const T zm = weno_side<T, FAST>(w, p.inv[2], false, p.fp64_kinks);
        if (KIND == kStageReinit) {
          const T pc = p.use_phi0 == 1 ? __ldg(p.aux0 + o) : w[3];
          L = reinit_cell(pc, xp, yp, zp, xm, ym, zm, p.dx_sq, p.use_phi0 == 1);
        } else {
          // LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS (:209-231)
          const T f = __ldg(p.aux0 + o);
          L = T(0);
          if (fabsT(f) >= Consts<T>::zero_tol)
            L = T(0) - f * sqrtT(godunov_sq2(f, xp, yp, zp, xm, ym, zm));
          if (KIND == kStageNormalRhs) {
            // LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT per-cell speed (FP64)
            const double cx = fmax2(fabs((double)xp), fabs((double)xm));
            const double cy = fmax2(fabs((double)yp), fabs((double)ym));
            const double cz = fmax2(fabs((double)zp), fabs((double)zm));
            const double ng = sqrt(cx * cx + cy * cy + cz * cz + (double)p.dx_sq);
            const double h = fabs((double)f) / ng *
                             (cx * (double)p.inv[0] + cy * (double)p.inv[1] +
                              cz * (double)p.inv[2]);
            hmax = (h > hmax) ? h : hmax;
          }
        }
      }
      if (KIND == kStageNormalRhs) {
        p.rhs_out[o] = L;
      } else {
        const T uc = (p.rk_kind == 1) ? T(0) : __ldg(p.phi_n + o);
        p.out[o] = rk_combine(p.rk_kind, uc, w[3], L, dt);
      }
    }
    __syncthreads();
  }
  if (KIND == kStageNormalRhs) {
    // block maximum with the reference's "if (h > m) m = h" comparison
    __shared__ double red[TX * TY / 32];
    double m = hmax;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double o2 = __shfl_xor_sync(0xffffffffu, m, off);
      m = (o2 > m) ? o2 : m;
    }
    const int lane = (ty * TX + tx) & 31, wid = (ty * TX + tx) >> 5;
    if (lane == 0) red[wid] = m;
    __syncthreads();
    if (wid == 0) {
      m = (lane < TX * TY / 32) ? red[lane] : -1.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double o2 = __shfl_xor_sync(0xffffffffu, m, off);
        m = (o2 > m) ? o2 : m;
      }
      if (lane == 0)
        p.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = m;
    }
  }
}

}  // namespace lsmgpu
