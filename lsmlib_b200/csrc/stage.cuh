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
  kStageNormalRhs = 3, // normal speed, writes L(phi) and CFL maxima only
  kStageAdvectConst = 4, // constant velocity vel_const: upwind WENO5, -V.grad
  kStageDeformation = 5  // LeVeque's deformation field from sine tables
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
  FaceConst<T> fk[3];  // face_const(inv[d]): the face-shared kernels' WENO5 constants
  T dx_sq;             // max(dx,dy,dz)^2 (reinit sign, CFL)
  const double* dt_dev;
  double dt;
  int rk_kind;         // 1, 22, 32, 33 (see rk_update)
  int use_phi0;
  int fp64_policy;     // FP32 form: kFp64Kinks | kFp64Sign (see below)
  unsigned sr_seed;    // FP32 form: nonzero = stochastic rounding of out
  T vel_const[3];      // kStageAdvectConst: the grid's constant velocity
  // kStageDeformation: sin(pi x), sin(2 pi x) of the fill-box cell centres
  // of axis d at defo_tab + defo_off[d] (n_d values each, one after the
  // other) and g(t + c dt) at *g_dev
  const double* defo_tab;
  int defo_off[3];
  const double* g_dev;
  // FP64 band of an FP32 workspace (k_stage_pairs_up): tile_fp64[tile], tiles
  // numbered in launch order, says which precision computes a tile; such a
  // launch computes only the tiles whose flag equals tile_want, and writes
  // each output cell also into out_alt, the same stage output in the other
  // precision (FP32 rounded to nearest, or FP64 widened exactly)
  const unsigned char* tile_fp64 = nullptr;
  unsigned tile_want = 0u;
  void* out_alt = nullptr;
};

// LeVeque's 3D deformation velocity of a cell from its sine values and g,
// in the expression order of the reference-layout velocity arrays
// (u = 2 sin^2(pi x) sin(2 pi y) sin(2 pi z) g, v = -sin(2 pi x) sin^2(pi y)
// sin(2 pi z) g, w = -sin(2 pi x) sin(2 pi y) sin^2(pi z) g); products only,
// so no FMA contraction can change them.
struct DeformSines {
  double sx, s2x, sy, s2y, sz, s2z;
};
template <typename T>
__device__ __forceinline__ void deformation_velocity(const DeformSines& s, double g,
                                                     T& u, T& v, T& w) {
  u = (T)(2.0 * s.sx * s.sx * s.s2y * s.s2z * g);
  v = (T)(-s.s2x * s.sy * s.sy * s.s2z * g);
  w = (T)(-s.s2x * s.s2y * s.sz * s.sz * g);
}

// FP64 parts of the FP32 form: kFp64Kinks recomputes in FP64 the WENO5
// stencils whose smoothness indicators differ by more than a factor 1e3;
// kFp64Sign evaluates the smoothed sign of the reinitialization RHS in FP64;
// kStochRound forms the Runge-Kutta combination in FP64 and rounds it to
// FP32 stochastically (sr_float).
// kFp64Band (drivers of an FP32 workspace in fast mode) computes the tiles
// near the interface in FP64 from FP64 copies of the stage arrays.
constexpr int kFp64Kinks = 1, kFp64Sign = 2, kStochRound = 4, kFp64Band = 8;

// the other precision's copy of a stage output (FP64 band form)
__device__ __forceinline__ void store_alt(void* alt, long o, double v) {
  static_cast<float*>(alt)[o] = (float)v;
}
__device__ __forceinline__ void store_alt(void* alt, long o, float v) {
  static_cast<double*>(alt)[o] = (double)v;
}

template <typename T>
__device__ __forceinline__ T rk_combine(int kind, T uc, T us, T r, T dt) {
  switch (kind) {
    case 22: return T(0.5) * (uc + us + dt * r);
    case 32: return T(0.75) * uc + T(0.25) * (us + dt * r);
    case 33: return (T(1) / T(3)) * uc + (T(2) / T(3)) * (us + dt * r);
    default: return us + dt * r;
  }
}

// the stage output of cell offset o: the Runge-Kutta combination, in the FP32
// form with stochastic rounding when the launch has a seed
template <typename T>
__device__ __forceinline__ T stage_out(const StageParams<T>& p, long o, T uc, T us,
                                       T r, T dt) {
  if (sizeof(T) == 4 && p.sr_seed != 0u) {
    const double dtd = p.dt_dev ? *p.dt_dev : p.dt;
    const double v = rk_combine<double>(p.rk_kind, uc, us, r, dtd);
    return (T)sr_float(v, sr_hash((unsigned)o * 0x9e3779b9u ^ p.sr_seed));
  }
  return rk_combine(p.rk_kind, uc, us, r, dt);
}

// Boundary kinds per face f (0..5 = x-lo, x-hi, y-lo, y-hi, z-lo, z-hi) in
// StageParams::bc_mask: bit f = linear extrapolation
// (lsm_boundary_conditions3d.f:46-170), bit 8+f = copy extrapolation
// (homogeneous Neumann, :352-463), bit 16+f = periodic; no bit = the ghost
// cells stored in the array.
constexpr unsigned kBcLinear = 0x3fu, kBcCopy = 0x3fu << 8, kBcPeriodic = 0x3fu << 16;

// phi at (i,j,k) where at most one coordinate may lie outside the domain box
template <typename T>
__device__ __forceinline__ T fetch_bc(const Grid3<const T>& g,
                                      const StageParams<T>& p, int i, int j,
                                      int k) {
  const unsigned m = p.bc_mask;
  if (m & kBcPeriodic) {
    const int nx = p.dom.hi[0] - p.dom.lo[0] + 1, ny = p.dom.hi[1] - p.dom.lo[1] + 1,
              nz = p.dom.hi[2] - p.dom.lo[2] + 1;
    if (i < p.dom.lo[0] && (m & (1u << 16))) return __ldg(g.ptr(i + nx, j, k));
    if (i > p.dom.hi[0] && (m & (2u << 16))) return __ldg(g.ptr(i - nx, j, k));
    if (j < p.dom.lo[1] && (m & (4u << 16))) return __ldg(g.ptr(i, j + ny, k));
    if (j > p.dom.hi[1] && (m & (8u << 16))) return __ldg(g.ptr(i, j - ny, k));
    if (k < p.dom.lo[2] && (m & (16u << 16))) return __ldg(g.ptr(i, j, k + nz));
    if (k > p.dom.hi[2] && (m & (32u << 16))) return __ldg(g.ptr(i, j, k - nz));
  }
  if (m & kBcCopy) {
    if (i < p.dom.lo[0] && (m & (1u << 8))) return __ldg(g.ptr(p.dom.lo[0], j, k));
    if (i > p.dom.hi[0] && (m & (2u << 8))) return __ldg(g.ptr(p.dom.hi[0], j, k));
    if (j < p.dom.lo[1] && (m & (4u << 8))) return __ldg(g.ptr(i, p.dom.lo[1], k));
    if (j > p.dom.hi[1] && (m & (8u << 8))) return __ldg(g.ptr(i, p.dom.hi[1], k));
    if (k < p.dom.lo[2] && (m & (16u << 8))) return __ldg(g.ptr(i, j, p.dom.lo[2]));
    if (k > p.dom.hi[2] && (m & (32u << 8))) return __ldg(g.ptr(i, j, p.dom.hi[2]));
  }
  const T* e;
  long inward;
  int dist;
  if (i < p.dom.lo[0] && (p.bc_mask & 1u)) {
    e = g.ptr(p.dom.lo[0], j, k); inward = 1; dist = p.dom.lo[0] - i;
  } else if (i > p.dom.hi[0] && (p.bc_mask & 2u)) {
    e = g.ptr(p.dom.hi[0], j, k); inward = -1; dist = i - p.dom.hi[0];
  } else if (j < p.dom.lo[1] && (p.bc_mask & 4u)) {
    e = g.ptr(i, p.dom.lo[1], k); inward = g.sy; dist = p.dom.lo[1] - j;
  } else if (j > p.dom.hi[1] && (p.bc_mask & 8u)) {
    e = g.ptr(i, p.dom.hi[1], k); inward = -g.sy; dist = j - p.dom.hi[1];
  } else if (k < p.dom.lo[2] && (p.bc_mask & 16u)) {
    e = g.ptr(i, j, p.dom.lo[2]); inward = g.sz; dist = p.dom.lo[2] - k;
  } else if (k > p.dom.hi[2] && (p.bc_mask & 32u)) {
    e = g.ptr(i, j, p.dom.hi[2]); inward = -g.sz; dist = k - p.dom.hi[2];
  } else {
    return __ldg(g.ptr(i, j, k));
  }
  const T e0 = __ldg(e), e1 = __ldg(e + inward);
  const T slope = e0 - e1;
  return e0 + slope * (T)dist;
}

// One-sided WENO5 from seven consecutive phi values w[0..6] = phi(c-3..c+3).
template <typename T, bool FAST>
__device__ __forceinline__ T weno_minus7(const T* w, T inv) {
  if (FAST)
    return weno5_side_fast(w[1] - w[0], w[2] - w[1], w[3] - w[2], w[4] - w[3], w[5] - w[4],
                           inv);
  const T v1 = (w[1] - w[0]) * inv, v2 = (w[2] - w[1]) * inv,
          v3 = (w[3] - w[2]) * inv, v4 = (w[4] - w[3]) * inv,
          v5 = (w[5] - w[4]) * inv;
  return weno5_strict(v1, v2, v3, v4, v5);
}
template <typename T, bool FAST>
__device__ __forceinline__ T weno_plus7(const T* w, T inv) {
  if (FAST)
    return weno5_side_fast(w[6] - w[5], w[5] - w[4], w[4] - w[3], w[3] - w[2], w[2] - w[1],
                           inv);
  const T v1 = (w[6] - w[5]) * inv, v2 = (w[5] - w[4]) * inv,
          v3 = (w[4] - w[3]) * inv, v4 = (w[3] - w[2]) * inv,
          v5 = (w[2] - w[1]) * inv;
  return weno5_strict(v1, v2, v3, v4, v5);
}

// FP32 form: the same values, with kink stencils recomputed in FP64 from the
// FP32 phi values (the kink test is scale-free, so it reads the undivided
// differences).
template <typename T, bool FAST>
__device__ __forceinline__ T weno_side(const T* w, T inv, bool plus,
                                       bool fp64_kinks) {
  if (sizeof(T) == 4 && fp64_kinks) {
    const T v1 = plus ? w[6] - w[5] : w[1] - w[0];
    const T v2 = plus ? w[5] - w[4] : w[2] - w[1];
    const T v3 = plus ? w[4] - w[3] : w[3] - w[2];
    const T v4 = plus ? w[3] - w[2] : w[4] - w[3];
    const T v5 = plus ? w[2] - w[1] : w[5] - w[4];
    if (weno5_is_kink(v1, v2, v3, v4, v5)) {
      double wd[7];
#pragma unroll
      for (int m = 0; m < 7; m++) wd[m] = (double)w[m];
      const double id = (double)inv;
      return (T)(plus ? weno_plus7<double, true>(wd, id)
                      : weno_minus7<double, true>(wd, id));
    }
    return weno5_side_fast(v1, v2, v3, v4, v5, inv);
  }
  return plus ? weno_plus7<T, FAST>(w, inv) : weno_minus7<T, FAST>(w, inv);
}

// Godunov |grad phi|^2 of the normal-speed term
// (lsm_level_set_evolution3d.f.in:209-231): per axis, for vn > 0,
// max(max(phi^-, 0)^2, min(phi^+, 0)^2).  Both operands are squares of
// non-negative numbers (max(phi^-, 0) and -min(phi^+, 0)), and rounding is
// monotone, so the larger square is the square of the larger of the two:
// max(phi^-, -phi^+, 0)^2, the same value in two comparisons and one product
// instead of three and two (a zero's sign, the only difference, squares away).
template <typename T>
__device__ __forceinline__ T godunov_sq2(T vn, T xp, T yp, T zp, T xm, T ym,
                                         T zm) {
  const T z = T(0);
  T ax, ay, az;
  if (vn > z) {
    ax = fmax2(fmax2(xm, -xp), z); ay = fmax2(fmax2(ym, -yp), z); az = fmax2(fmax2(zm, -zp), z);
  } else {
    ax = fmax2(fmax2(-xm, xp), z); ay = fmax2(fmax2(-ym, yp), z); az = fmax2(fmax2(-zm, zp), z);
  }
  T s = ax * ax;
  s = s + ay * ay;
  s = s + az * az;
  return s;
}

// reinitialization RHS of one cell (lsm_reinitialization3d.f.in:158-199,
// :218-256); with fp64_sign the FP32 form evaluates the smoothed sign in FP64.
// FASTM: the divisions by square roots and the square root of |grad phi|^2
// through rsqrt_nr (FMA arithmetic; the strict form keeps the reference's
// correctly rounded division and square root).
template <typename T, bool FASTM = false>
__device__ __forceinline__ T reinit_cell(T pc, T xp, T yp, T zp, T xm, T ym,
                                         T zm, T dx_sq, bool use0,
                                         bool fp64_sign) {
  const T z = T(0);
  T gp[3] = {xp, yp, zp}, gm[3] = {xm, ym, zm}, gs[3];
  // per axis max(max(-+phi^+, 0), max(+-phi^-, 0)) as max(-+phi^+, +-phi^-, 0):
  // the same value (but for a zero's sign, which squares away) in two
  // comparisons instead of three
#pragma unroll
  for (int d = 0; d < 3; d++)
    gs[d] = pc > z ? fmax2(fmax2(-gp[d], gm[d]), z) : fmax2(fmax2(gp[d], -gm[d]), z);
  // FP64 build's zero_tol for both precisions (see stage_zero_tol)
  if (!(fabsT(pc) >= T(1.0e-11))) return z;
  const T nsq = gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2];
  if (sizeof(T) == 4 && fp64_sign) {
    const double pd = pc, nd = nsq, dd = dx_sq;
    if (FASTM) {
      // |pc| >= 1e-11, so the sums are positive normal numbers
      const double sgn = pd * rsqrt_nr(use0 ? pd * pd + dd : pd * pd + nd * dd);
      return (T)(sgn * (1.0 - sqrt_nr(nd)));
    }
    const double sgn = use0 ? pd / sqrt(pd * pd + dd) : pd / sqrt(pd * pd + nd * dd);
    return (T)(sgn * (1.0 - sqrt(nd)));
  }
  if (FASTM) {
    const T sgn = pc * rsqrt_nr(use0 ? pc * pc + dx_sq : pc * pc + nsq * dx_sq);
    return sgn * (T(1) - sqrt_nr(nsq));
  }
  const T sgn = use0 ? pc / sqrtT(pc * pc + dx_sq)
                     : pc / sqrtT(pc * pc + nsq * dx_sq);
  return sgn * (T(1) - sqrtT(nsq));
}

// Zero tolerance of the fused stages.  The FP32 form keeps the FP64 build's
// value (configure.ac:268) so that its decisions track the FP64 reference;
// the reference's single-precision build uses 1e-5 (configure.ac:265), which
// would switch the reinitialization RHS off at |phi| < 1e-5 where the FP64
// build keeps it (a difference of a whole pseudo-step dt at such cells).
template <typename T>
__device__ __forceinline__ T stage_zero_tol() { return T(1.0e-11); }

// plus and minus WENO5 of one axis from w[0..6] = phi(c-3..c+3)
template <typename T, bool FAST>
__device__ __forceinline__ void weno_axis(const T* w, T inv, bool kink64, T& vp,
                                          T& vm) {
  if (FAST || sizeof(T) == 4) {
    if (sizeof(T) == 4 && kink64) weno5_pm_fast<T, true>(w, inv, vp, vm);
    else weno5_pm_fast<T, false>(w, inv, vp, vm);
  } else {
    vp = weno_plus7<T, false>(w, inv);
    vm = weno_minus7<T, false>(w, inv);
  }
}

// one side only (upwind derivative)
template <typename T, bool FAST>
__device__ __forceinline__ T weno_upwind_side(const T* w, T inv, bool plus,
                                              bool kink64) {
  if (FAST || sizeof(T) == 4) return weno_side<T, true>(w, inv, plus, kink64);
  return plus ? weno_plus7<T, false>(w, inv) : weno_minus7<T, false>(w, inv);
}

// One tile of a fused stage: TX x TY cells (tile bx, by) marched over planes
// [bz*TZ, bz*TZ + TZ) of the fill box.  ``tile`` holds two shared planes:
// plane k is written into buffer (k-kb)&1 while the other buffer may still be
// read by slower threads of the previous plane.  Returns the tile's largest
// CFL speed for kStageNormalRhs (-1 otherwise).  The caller synchronises the
// block before reusing ``tile``.
// STAGING is the halo-staging schedule of the x/y stencils: 0 stages each
// plane with its 3-cell side strips in shared memory (two barriers per
// plane); 1 reads the x and y neighbours straight from global memory through
// L1 (no shared plane, no barrier; neighbouring threads share the cache
// lines).  The batched autotuner picks one per batch.
template <typename T, int KIND, bool FAST, int TX, int TY, int TZ, int STAGING = 0>
__device__ __forceinline__ double stage_tile(const StageParams<T>& p, int bx,
                                             int by, int bz,
                                             T (*tile)[TY + 6][TX + 6]) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = p.fb.lo[0] + bx * TX + tx;
  const int j = p.fb.lo[1] + by * TY + ty;
  const int kb = p.fb.lo[2] + bz * TZ;
  const int ke = min(kb + TZ - 1, p.fb.hi[2]);
  const bool act = (i <= p.fb.hi[0]) && (j <= p.fb.hi[1]);
  const Grid3<const T> phi = make_grid(p.phi_s, p.gb);
  const long sy = p.gb.sy(), sz = p.gb.sz();
  const long base0 = -((long)p.gb.lo[0] + sy * p.gb.lo[1] + sz * p.gb.lo[2]);
  const T dt = p.dt_dev ? (T)(*p.dt_dev) : (T)p.dt;
  // Boundary values are generated only by tiles whose stencil reaches past
  // the domain box; every other tile loads directly (block-uniform test).
  const int xlo = p.fb.lo[0] + bx * TX - 3, xhi = min(p.fb.lo[0] + bx * TX + TX - 1, p.fb.hi[0]) + 3;
  const int ylo = p.fb.lo[1] + by * TY - 3, yhi = min(p.fb.lo[1] + by * TY + TY - 1, p.fb.hi[1]) + 3;
  const bool inside = xlo >= p.dom.lo[0] && xhi <= p.dom.hi[0] && ylo >= p.dom.lo[1] &&
                      yhi <= p.dom.hi[1] && kb - 3 >= p.dom.lo[2] &&
                      ke + 3 <= p.dom.hi[2];
  const bool need_bc = p.bc_mask != 0u && !inside;
  const bool kink64 = (p.fp64_policy & kFp64Kinks) != 0;
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
  const int tcol = (tx < 3) ? tx : tx + 6;
  const int trow = (ty < 3) ? ty : ty + 6;

  auto ld = [&](int a, int b, int c) -> T {
    return need_bc ? fetch_bc(phi, p, a, b, c) : __ldg(phi.ptr(a, b, c));
  };

  // registers of the plane to be written next: the new top of the z window
  // (active threads) or the own cell (halo threads), and the strip cells
  T nx_c = T(0), nx_hx = T(0), nx_hy = T(0);
  auto prefetch = [&](int k) {
    if (act) nx_c = ld(i, j, k + 3);
    else if (STAGING == 0 && ctr_halo) nx_c = ld(i, j, k);
    if (STAGING == 0 && has_hx) nx_hx = ld(hx, j, k);
    if (STAGING == 0 && has_hy) nx_hy = ld(i, hj, k);
  };

  T w[7];
  if (act) {
#pragma unroll
    for (int m = 0; m < 6; m++) w[m + 1] = ld(i, j, kb - 3 + m);
  }
  prefetch(kb);
  for (int k = kb; k <= ke; ++k) {
    const int buf = (k - kb) & 1;
    if (act) {
#pragma unroll
      for (int m = 0; m < 6; m++) w[m] = w[m + 1];
      w[6] = nx_c;
      if constexpr (STAGING == 0) tile[buf][ty + 3][tx + 3] = w[3];
    } else if (STAGING == 0 && ctr_halo) {
      tile[buf][ty + 3][tx + 3] = nx_c;
    }
    if constexpr (STAGING == 0) {
      if (has_hx) tile[buf][ty + 3][tcol] = nx_hx;
      if (has_hy) tile[buf][trow][tx + 3] = nx_hy;
      __syncthreads();
    }
    if (k < ke) prefetch(k + 1);
    if (act) {
      const long o = base0 + (long)i + sy * j + sz * k;
      // point loads of this cell, issued before the stencil arithmetic
      T a0 = T(0), a1 = T(0), a2 = T(0), uc = T(0);
      if (KIND == kStageAdvect) {
        a0 = __ldg(p.aux0 + o); a1 = __ldg(p.aux1 + o); a2 = __ldg(p.aux2 + o);
      } else if (KIND == kStageDeformation) {
        const int nx = p.fb.hi[0] - p.fb.lo[0] + 1, ny = p.fb.hi[1] - p.fb.lo[1] + 1,
                  nz = p.fb.hi[2] - p.fb.lo[2] + 1;
        const double* tx_ = p.defo_tab + p.defo_off[0] + (i - p.fb.lo[0]);
        const double* ty_ = p.defo_tab + p.defo_off[1] + (j - p.fb.lo[1]);
        const double* tz_ = p.defo_tab + p.defo_off[2] + (k - p.fb.lo[2]);
        DeformSines s;
        s.sx = __ldg(tx_); s.s2x = __ldg(tx_ + nx);
        s.sy = __ldg(ty_); s.s2y = __ldg(ty_ + ny);
        s.sz = __ldg(tz_); s.s2z = __ldg(tz_ + nz);
        deformation_velocity(s, __ldg(p.g_dev), a0, a1, a2);
      } else if (KIND == kStageAdvectConst) {
        a0 = p.vel_const[0]; a1 = p.vel_const[1]; a2 = p.vel_const[2];
      } else if (KIND == kStageNormal || KIND == kStageNormalRhs ||
                 (KIND == kStageReinit && p.use_phi0 == 1)) {
        a0 = __ldg(p.aux0 + o);
      }
      if (KIND != kStageNormalRhs && p.rk_kind != 1) uc = __ldg(p.phi_n + o);
      T wx[7], wy[7];
      if constexpr (STAGING == 0) {
#pragma unroll
        for (int m = 0; m < 7; m++) {
          wx[m] = tile[buf][ty + 3][tx + m];
          wy[m] = tile[buf][ty + m][tx + 3];
        }
      } else {
#pragma unroll
        for (int m = 0; m < 7; m++) {
          wx[m] = m == 3 ? w[3] : ld(i - 3 + m, j, k);
          wy[m] = m == 3 ? w[3] : ld(i, j - 3 + m, k);
        }
      }
      const T ztol = stage_zero_tol<T>();
      T L;
      if (KIND == kStageAdvect || KIND == kStageAdvectConst || KIND == kStageDeformation) {
        // LSM3D_UPWIND_HJ_WENO5 + LSM3D_ADD_ADVECTION_TERM_TO_LSE_RHS
        T gx = T(0), gy = T(0), gz = T(0);
        if (!(fabsT(a0) < ztol))
          gx = weno_upwind_side<T, FAST>(wx, p.inv[0], !(a0 > T(0)), kink64);
        if (!(fabsT(a1) < ztol))
          gy = weno_upwind_side<T, FAST>(wy, p.inv[1], !(a1 > T(0)), kink64);
        if (!(fabsT(a2) < ztol))
          gz = weno_upwind_side<T, FAST>(w, p.inv[2], !(a2 > T(0)), kink64);
        L = T(0) - (a0 * gx + a1 * gy + a2 * gz);
      } else {
        T xp, xm, yp, ym, zp, zm;
        weno_axis<T, FAST>(wx, p.inv[0], kink64, xp, xm);
        weno_axis<T, FAST>(wy, p.inv[1], kink64, yp, ym);
        weno_axis<T, FAST>(w, p.inv[2], kink64, zp, zm);
        if (KIND == kStageReinit) {
          const T pc = p.use_phi0 == 1 ? a0 : w[3];
          L = reinit_cell(pc, xp, yp, zp, xm, ym, zm, p.dx_sq, p.use_phi0 == 1,
                          (p.fp64_policy & kFp64Sign) != 0);
        } else {
          // LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS (:209-231)
          const T f = a0;
          L = T(0);
          if (fabsT(f) >= ztol)
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
        p.out[o] = stage_out(p, o, uc, w[3], L, dt);
      }
    }
  }
  return hmax;
}

// Right-hand side of the two-sided kinds (normal speed, reinitialization)
// from the six one-sided derivatives; accumulates the CFL speed of
// kStageNormalRhs into hmax.  FASTM as for reinit_cell.
template <typename T, int KIND, bool FASTM = false>
__device__ __forceinline__ T two_sided_rhs(const StageParams<T>& p, T a0, T pc,
                                           T xp, T yp, T zp, T xm, T ym, T zm,
                                           double& hmax) {
  if (KIND == kStageReinit) {
    const T s = p.use_phi0 == 1 ? a0 : pc;
    return reinit_cell<T, FASTM>(s, xp, yp, zp, xm, ym, zm, p.dx_sq, p.use_phi0 == 1,
                                 (p.fp64_policy & kFp64Sign) != 0);
  }
  // LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS (:209-231)
  const T f = a0;
  T L = T(0);
  if (fabsT(f) >= stage_zero_tol<T>()) {
    const T g2 = godunov_sq2(f, xp, yp, zp, xm, ym, zm);
    L = T(0) - f * (FASTM ? sqrt_nr(g2) : sqrtT(g2));
  }
  if (KIND == kStageNormalRhs) {
    // LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT per-cell speed (FP64)
    const double cx = fmax2(fabs((double)xp), fabs((double)xm));
    const double cy = fmax2(fabs((double)yp), fabs((double)ym));
    const double cz = fmax2(fabs((double)zp), fabs((double)zm));
    const double n2 = cx * cx + cy * cy + cz * cz + (double)p.dx_sq;
    const double sum = cx * (double)p.inv[0] + cy * (double)p.inv[1] + cz * (double)p.inv[2];
    // n2 >= dx_sq > 0
    const double h = FASTM ? fabs((double)f) * rsqrt_nr(n2) * sum
                           : fabs((double)f) / sqrt(n2) * sum;
    hmax = (h > hmax) ? h : hmax;
  }
  return L;
}

// value of the lane to the left (lane 0 gets its own back)
template <typename T>
__device__ __forceinline__ T shfl_up_T(T v) {
  return __shfl_up_sync(0xffffffffu, v, 1);
}

template <typename T>
__device__ __forceinline__ void face_pm(const T* u, T inv, bool kink64, T& vp,
                                        T& vm) {
  if (sizeof(T) == 4 && kink64) weno5_face<T, true>(u, inv, vp, vm);
  else weno5_face<T, false>(u, inv, vp, vm);
}

// The two-sided kinds in the FMA/FP32 arithmetic, one WENO5 weight
// evaluation per cell face instead of one per cell side (weno5_face): the
// thread of cell c evaluates the face c+1/2 of each axis, giving phi^+(c)
// and phi^-(c+1).  phi^-(c) comes from the neighbour that owns face c-1/2:
// along x the lane to the left (warp shuffle; a tile row is one warp), along
// y the row below (shared memory), along z the previous plane of the march
// (a register).  The faces in front of the first cell of each row, column
// and z run are evaluated once more (rows by warp 0, columns by the last
// warp, z at the first plane).  Tile staging, boundary values and prefetch
// are those of stage_tile.
template <typename T, int KIND, int TX, int TY, int TZ>
__device__ __forceinline__ double stage_tile_faces(const StageParams<T>& p, int bx,
                                                   int by, int bz,
                                                   T (*tile)[TY + 6][TX + 6],
                                                   T (*fy)[TX], T* fx) {
  static_assert(TX == 32, "a tile row is one warp");
  static_assert(TY <= 32, "row-start faces are spread over one warp");
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = p.fb.lo[0] + bx * TX + tx;
  const int j = p.fb.lo[1] + by * TY + ty;
  const int kb = p.fb.lo[2] + bz * TZ;
  const int ke = min(kb + TZ - 1, p.fb.hi[2]);
  const bool act = (i <= p.fb.hi[0]) && (j <= p.fb.hi[1]);
  const Grid3<const T> phi = make_grid(p.phi_s, p.gb);
  const long sy = p.gb.sy(), sz = p.gb.sz();
  const long base0 = -((long)p.gb.lo[0] + sy * p.gb.lo[1] + sz * p.gb.lo[2]);
  const T dt = p.dt_dev ? (T)(*p.dt_dev) : (T)p.dt;
  const int xlo = p.fb.lo[0] + bx * TX - 3, xhi = min(p.fb.lo[0] + bx * TX + TX - 1, p.fb.hi[0]) + 3;
  const int ylo = p.fb.lo[1] + by * TY - 3, yhi = min(p.fb.lo[1] + by * TY + TY - 1, p.fb.hi[1]) + 3;
  const bool inside = xlo >= p.dom.lo[0] && xhi <= p.dom.hi[0] && ylo >= p.dom.lo[1] &&
                      yhi <= p.dom.hi[1] && kb - 3 >= p.dom.lo[2] &&
                      ke + 3 <= p.dom.hi[2];
  const bool need_bc = p.bc_mask != 0u && !inside;
  const bool kink64 = (p.fp64_policy & kFp64Kinks) != 0;
  double hmax = -1.0;

  const int hi0 = p.fb.hi[0], hi1 = p.fb.hi[1];
  const bool ctr_halo = !act && i <= hi0 + 3 && j <= hi1 + 3 && !(i > hi0 && j > hi1);
  const int hx = (tx < 3) ? (i - 3) : (i + 3);
  const bool has_hx = (j <= hi1) && ((tx < 3) || (tx >= TX - 3 && i <= hi0));
  const int hj = (ty < 3) ? (j - 3) : (j + 3);
  const bool has_hy = (i <= hi0) && ((ty < 3) || (ty >= TY - 3 && j <= hi1));
  const int tcol = (tx < 3) ? tx : tx + 6;
  const int trow = (ty < 3) ? ty : ty + 6;
  // row-start face of row tx (warp 0) / column-start face of column tx
  // (last warp): is that row / column part of the fill box?
  const bool row_start = ty == 0 && tx < TY && p.fb.lo[1] + by * TY + tx <= hi1;
  const bool col_start = ty == TY - 1 && i <= hi0;

  auto ld = [&](int a, int b, int c) -> T {
    return need_bc ? fetch_bc(phi, p, a, b, c) : __ldg(phi.ptr(a, b, c));
  };
  T nx_c = T(0), nx_hx = T(0), nx_hy = T(0);
  auto prefetch = [&](int k) {
    if (act) nx_c = ld(i, j, k + 3);
    else if (ctr_halo) nx_c = ld(i, j, k);
    if (has_hx) nx_hx = ld(hx, j, k);
    if (has_hy) nx_hy = ld(i, hj, k);
  };

  T w[7];
  if (act) {
#pragma unroll
    for (int m = 0; m < 6; m++) w[m + 1] = ld(i, j, kb - 3 + m);
  }
  T zm_run = T(0);  // phi_z^-(k), from face k-1/2 of the previous plane
  prefetch(kb);
  for (int k = kb; k <= ke; ++k) {
    const int buf = (k - kb) & 1;
    if (act) {
#pragma unroll
      for (int m = 0; m < 6; m++) w[m] = w[m + 1];
      w[6] = nx_c;
      tile[buf][ty + 3][tx + 3] = w[3];
    } else if (ctr_halo) {
      tile[buf][ty + 3][tx + 3] = nx_c;
    }
    if (has_hx) tile[buf][ty + 3][tcol] = nx_hx;
    if (has_hy) tile[buf][trow][tx + 3] = nx_hy;
    __syncthreads();
    if (k < ke) prefetch(k + 1);
    const long o = base0 + (long)i + sy * j + sz * k;
    T a0 = T(0), uc = T(0);
    T xp = T(0), xm_next = T(0), yp = T(0), zp = T(0), zm_next = T(0);
    if (act) {
      if (KIND == kStageNormal || KIND == kStageNormalRhs ||
          (KIND == kStageReinit && p.use_phi0 == 1))
        a0 = __ldg(p.aux0 + o);
      if (KIND != kStageNormalRhs && p.rk_kind != 1) uc = __ldg(p.phi_n + o);
      T u[6], ym_next;
#pragma unroll
      for (int m = 0; m < 6; m++) u[m] = tile[buf][ty + 3][tx + 1 + m];
      face_pm(u, p.inv[0], kink64, xp, xm_next);
#pragma unroll
      for (int m = 0; m < 6; m++) u[m] = tile[buf][ty + 1 + m][tx + 3];
      face_pm(u, p.inv[1], kink64, yp, ym_next);
      if (ty + 1 < TY) fy[ty + 1][tx] = ym_next;
      if (k == kb) {
        T unused;
        face_pm(w, p.inv[2], kink64, unused, zm_run);
      }
      face_pm(w + 1, p.inv[2], kink64, zp, zm_next);
    }
    const T xm_left = shfl_up_T(xm_next);
    if (row_start) {
      T u[6], unused;
#pragma unroll
      for (int m = 0; m < 6; m++) u[m] = tile[buf][tx + 3][m];
      face_pm(u, p.inv[0], kink64, unused, fx[tx]);
    }
    if (col_start) {
      T u[6], unused;
#pragma unroll
      for (int m = 0; m < 6; m++) u[m] = tile[buf][m][tx + 3];
      face_pm(u, p.inv[1], kink64, unused, fy[0][tx]);
    }
    __syncthreads();
    if (act) {
      const T xm = tx == 0 ? fx[ty] : xm_left;
      const T ym = fy[ty][tx];
      const T zm = zm_run;
      zm_run = zm_next;
      const T L = two_sided_rhs<T, KIND>(p, a0, w[3], xp, yp, zp, xm, ym, zm, hmax);
      if (KIND == kStageNormalRhs) p.rhs_out[o] = L;
      else p.out[o] = stage_out(p, o, uc, w[3], L, dt);
    }
  }
  return hmax;
}

template <typename T> struct Pair2;
template <> struct Pair2<double> { using type = double2; };
template <> struct Pair2<float> { using type = float2; };

// The face-shared two-sided kinds with two cells per thread: thread (t, ty)
// of a TX/2 x TY block owns the cells x0+2t and x0+2t+1 of row j0+ty and
// marches them along z.  Against one cell per thread this gives every
// thread six independent face evaluations per plane (the FP64 dependency
// chains of one cell no longer wait on each other), and the pair reads its
// x stencil (7 values for its two faces) and both y columns with 16-byte
// shared loads: the tile's x column of cell x is x - x0 + 4, so each pair
// starts on an even column.  The faces in front of each row are evaluated
// by row 0, those in front of each column by the last two rows (one column
// each) -- one inlined evaluation for both, from a strided tile read -- and
// the z face in front of the march before it starts.
// The kernel reads every ghost cell as stored (k_face_ghosts writes the
// boundary values first) and instantiates one face routine (K64: the FP32
// form's FP64 kink recomputation), so that its loop holds seven face
// evaluations and nothing else of size: its instruction footprint, not the
// arithmetic, limited a version with boundary loads and both face routines
// inlined (ncu: no_instruction stalls 4.1 per issue against 0.9).
// Everything else -- roles of the halo cells in partial tiles, the face
// owner of phi^- along each axis, the right-hand sides -- is that of
// stage_tile_faces.
constexpr int kPairPX = 4;

template <typename T, bool K64, bool LMAX = false>
__device__ __forceinline__ void face_pm_t(const T* u, const FaceConst<T>& k, T& vp, T& vm) {
  weno5_face<T, sizeof(T) == 4 && K64, LMAX>(u, k, vp, vm);
}

template <typename T, int KIND, bool K64, int TX, int TY, int TZ>
__device__ __forceinline__ double stage_tile_pairs(const StageParams<T>& p, int bx, int by,
                                                   int bz, T (*tile)[TY + 6][TX + 8],
                                                   T (*fy)[TX], T* fx) {
  using T2 = typename Pair2<T>::type;
  static_assert(TX == 32, "a tile row is one half-warp of pairs");
  static_assert(TY <= TX / 2, "row-start faces are spread over one row of threads");
  static_assert(TY >= 3, "row 0 and the last two rows are distinct");
  constexpr int NP = TX / 2;   // threads per row
  constexpr int PX = kPairPX;
  const int t = threadIdx.x, ty = threadIdx.y;
  const int x0 = p.fb.lo[0] + bx * TX, j0 = p.fb.lo[1] + by * TY;
  const int c0 = 2 * t;
  const int i0 = x0 + c0, i1 = i0 + 1;
  const int j = j0 + ty;
  const int kb = p.fb.lo[2] + bz * TZ;
  const int ke = min(kb + TZ - 1, p.fb.hi[2]);
  const int hi0 = p.fb.hi[0], hi1 = p.fb.hi[1];
  const bool rowin = j <= hi1;
  const bool act0 = rowin && i0 <= hi0, act1 = rowin && i1 <= hi0;
  const bool halo0 = !act0 && i0 <= hi0 + 3 && j <= hi1 + 3 && !(i0 > hi0 && j > hi1);
  const bool halo1 = !act1 && i1 <= hi0 + 3 && j <= hi1 + 3 && !(i1 > hi0 && j > hi1);
  const Grid3<const T> phi = make_grid(p.phi_s, p.gb);
  const long sy = p.gb.sy(), sz = p.gb.sz();
  const long base0 = -((long)p.gb.lo[0] + sy * p.gb.lo[1] + sz * p.gb.lo[2]);
  const T dt = p.dt_dev ? (T)(*p.dt_dev) : (T)p.dt;
  double hmax = -1.0;

  // x strips: cells x0-3, x0-2 (t = 0), x0-1 (t = 1) on the left; on the
  // right x0+TX, x0+TX+1 (t = NP-1) and x0+TX+2 (t = NP-2) where a cell of
  // the fill box is within 3 of them
  int hxa = 0, hxb = 0;
  bool has_a = false, has_b = false;
  if (rowin) {
    if (t == 0) { hxa = x0 - 3; hxb = x0 - 2; has_a = has_b = true; }
    else if (t == 1) { hxa = x0 - 1; has_a = true; }
    else if (t == NP - 1) {
      hxa = x0 + TX; hxb = x0 + TX + 1;
      has_a = hxa <= hi0 + 3; has_b = hxb <= hi0 + 3;
    } else if (t == NP - 2) { hxa = x0 + TX + 2; has_a = hxa <= hi0 + 3; }
  }
  const int cola = hxa - x0 + PX, colb = hxb - x0 + PX;
  // y strips: rows j0-3..j0-1 (ty < 3) and j+3 (ty >= TY-3, row in the fill
  // box), for the pair's cells that are fill-box columns
  const int hj = ty < 3 ? j0 - 3 + ty : j + 3;
  const bool has_hy = (ty < 3) || (ty >= TY - 3 && rowin);
  const bool hy0 = has_hy && i0 <= hi0, hy1 = has_hy && i1 <= hi0;
  const int trow = ty < 3 ? ty : ty + 6;
  // faces in front of rows (row 0, thread t < TY serves row t) and columns
  // (rows TY-2 and TY-1: column 2t and 2t+1 respectively)
  const bool row_start = ty == 0 && t < TY && j0 + t <= hi1;
  const int col_c = c0 + (ty == TY - 1 ? 1 : 0);
  const bool col_start = ty >= TY - 2 && x0 + col_c <= hi0;
  // the extra face as a strided read of buffer 0 (buffer 1 is one tile on)
  const bool xtra = row_start || col_start;
  const int xoff = row_start ? (t + 3) * (TX + 8) + PX - 3 : col_c + PX;
  const int xstride = row_start ? 1 : TX + 8;
  T* const xout = row_start ? &fx[t] : &fy[0][col_c];

  // 32-bit element offsets from the index-space origin (the launcher takes
  // this kernel only for arrays of fewer than 2^31 elements): the 64-bit
  // address arithmetic of every load was a twentieth of the integer work
  const T* P0 = p.phi_s + base0;
  const int isy = (int)sy, isz = (int)sz;
  auto ld = [&](int a, int b, int c) -> T { return __ldg(P0 + (a + isy * b + isz * c)); };
  // next plane's values: the window tops (active cells) or the own cells
  // (halo cells), and the strip cells
  T n0 = T(0), n1 = T(0), na = T(0), nb = T(0), ny0 = T(0), ny1 = T(0);
  auto prefetch = [&](int k) {
    if (act0) n0 = ld(i0, j, k + 3);
    else if (halo0) n0 = ld(i0, j, k);
    if (act1) n1 = ld(i1, j, k + 3);
    else if (halo1) n1 = ld(i1, j, k);
    if (has_a) na = ld(hxa, j, k);
    if (has_b) nb = ld(hxb, j, k);
    if (hy0) ny0 = ld(i0, hj, k);
    if (hy1) ny1 = ld(i1, hj, k);
  };

  // (a cell outside the fill box keeps zeros: the packed FP32 faces read
  // both windows)
  T w0[7] = {}, w1[7] = {};
  if (act0) {
#pragma unroll
    for (int m = 0; m < 6; m++) w0[m + 1] = ld(i0, j, kb - 3 + m);
  }
  if (act1) {
#pragma unroll
    for (int m = 0; m < 6; m++) w1[m + 1] = ld(i1, j, kb - 3 + m);
  }
  // phi_z^-(k) of each cell, from the face k-1/2 (first: the face in front
  // of the march, from phi(kb-3 .. kb+2))
  T zrun0 = T(0), zrun1 = T(0);
  if (act0) {
    T unused;
    face_pm_t<T, K64>(w0 + 1, p.fk[2], unused, zrun0);
    if (act1) face_pm_t<T, K64>(w1 + 1, p.fk[2], unused, zrun1);
  }
  prefetch(kb);
  for (int k = kb; k <= ke; ++k) {
    const int buf = (k - kb) & 1;
    T v0 = n0, v1 = n1;
    if (act0) {
#pragma unroll
      for (int m = 0; m < 6; m++) w0[m] = w0[m + 1];
      w0[6] = n0;
      v0 = w0[3];
    }
    if (act1) {
#pragma unroll
      for (int m = 0; m < 6; m++) w1[m] = w1[m + 1];
      w1[6] = n1;
      v1 = w1[3];
    }
    // the pair's own cells (a cell that is neither active nor halo is never
    // read, so it may hold anything)
    *reinterpret_cast<T2*>(&tile[buf][ty + 3][c0 + PX]) = T2{v0, v1};
    if (has_a) tile[buf][ty + 3][cola] = na;
    if (has_b) tile[buf][ty + 3][colb] = nb;
    if (hy0 || hy1) *reinterpret_cast<T2*>(&tile[buf][trow][c0 + PX]) = T2{ny0, ny1};
    __syncthreads();
    if (k < ke) prefetch(k + 1);
    const long o0 = base0 + (i0 + isy * j + isz * k);
    T a00 = T(0), a01 = T(0), uc0 = T(0), uc1 = T(0);
    T xp0 = T(0), xp1 = T(0), xm1 = T(0), xnext = T(0);
    T yp0 = T(0), yp1 = T(0), zp0 = T(0), zp1 = T(0), znx0 = T(0), znx1 = T(0);
    constexpr bool kAux = KIND == kStageNormal || KIND == kStageNormalRhs;
    if (act0) {
      if (kAux || (KIND == kStageReinit && p.use_phi0 == 1)) a00 = __ldg(p.aux0 + o0);
      if (KIND != kStageNormalRhs && p.rk_kind != 1) uc0 = __ldg(p.phi_n + o0);
    }
    if (act1) {
      if (kAux || (KIND == kStageReinit && p.use_phi0 == 1)) a01 = __ldg(p.aux0 + o0 + 1);
      if (KIND != kStageNormalRhs && p.rk_kind != 1) uc1 = __ldg(p.phi_n + o0 + 1);
    }
    if (act0) {
      // x: tile columns c0+2 .. c0+8 hold phi(x-2 .. x+4) of cell x = i0
      T u[7];
      const T2 q0 = *reinterpret_cast<const T2*>(&tile[buf][ty + 3][c0 + 2]);
      const T2 q1 = *reinterpret_cast<const T2*>(&tile[buf][ty + 3][c0 + 4]);
      const T2 q2 = *reinterpret_cast<const T2*>(&tile[buf][ty + 3][c0 + 6]);
      u[0] = q0.x; u[1] = q0.y; u[2] = q1.x; u[3] = q1.y; u[4] = q2.x; u[5] = q2.y;
      u[6] = tile[buf][ty + 3][c0 + 8];
      // y: both cells' columns, rows j-2 .. j+3
      T ya[6], yb[6];
#pragma unroll
      for (int m = 0; m < 6; m++) {
        const T2 q = *reinterpret_cast<const T2*>(&tile[buf][ty + 1 + m][c0 + PX]);
        ya[m] = q.x;
        yb[m] = q.y;
      }
      T ym0, ym1;
      if constexpr (sizeof(T) == 4 && !K64) {
        // FP32: the two faces of each axis in one packed evaluation
        float2 a[6], vp, vm;
#pragma unroll
        for (int m = 0; m < 6; m++) a[m] = make_float2(u[m], u[m + 1]);
        weno5_face2(a, p.inv[0], vp, vm);
        xp0 = vp.x; xp1 = vp.y; xm1 = vm.x; xnext = vm.y;
#pragma unroll
        for (int m = 0; m < 6; m++) a[m] = make_float2(ya[m], yb[m]);
        weno5_face2(a, p.inv[1], vp, vm);
        yp0 = vp.x; yp1 = vp.y; ym0 = vm.x; ym1 = vm.y;
#pragma unroll
        for (int m = 0; m < 6; m++) a[m] = make_float2(w0[m + 1], w1[m + 1]);
        weno5_face2(a, p.inv[2], vp, vm);
        zp0 = vp.x; zp1 = vp.y; znx0 = vm.x; znx1 = vm.y;
      } else {
        face_pm_t<T, K64, true>(u, p.fk[0], xp0, xm1);   // shares its eps maximum's
                                                          // inner part with the next
        face_pm_t<T, K64>(u + 1, p.fk[0], xp1, xnext);
        face_pm_t<T, K64>(ya, p.fk[1], yp0, ym0);
        face_pm_t<T, K64>(yb, p.fk[1], yp1, ym1);
        face_pm_t<T, K64>(w0 + 1, p.fk[2], zp0, znx0);
        if (act1) face_pm_t<T, K64>(w1 + 1, p.fk[2], zp1, znx1);
      }
      if (ty + 1 < TY) *reinterpret_cast<T2*>(&fy[ty + 1][c0]) = T2{ym0, ym1};
    }
    const T xm_left = __shfl_up_sync(0xffffffffu, xnext, 1, NP);
    if (xtra) {
      const T* xb = &tile[buf][0][0] + xoff;
      T u[6], unused;
#pragma unroll
      for (int m = 0; m < 6; m++) u[m] = xb[m * xstride];
      face_pm_t<T, K64>(u, face_const(row_start ? p.inv[0] : p.inv[1]), unused, *xout);
    }
    __syncthreads();
    if (act0) {
      const T2 ym = *reinterpret_cast<const T2*>(&fy[ty][c0]);
      const T xm0 = t == 0 ? fx[ty] : xm_left;
      const T L0 =
          two_sided_rhs<T, KIND, true>(p, a00, w0[3], xp0, yp0, zp0, xm0, ym.x, zrun0, hmax);
      zrun0 = znx0;
      if (KIND == kStageNormalRhs) p.rhs_out[o0] = L0;
      else p.out[o0] = stage_out(p, o0, uc0, w0[3], L0, dt);
      if (act1) {
        const T L1 = two_sided_rhs<T, KIND, true>(p, a01, w1[3], xp1, yp1, zp1, xm1, ym.y,
                                                  zrun1, hmax);
        zrun1 = znx1;
        if (KIND == kStageNormalRhs) p.rhs_out[o0 + 1] = L1;
        else p.out[o0 + 1] = stage_out(p, o0 + 1, uc1, w1[3], L1, dt);
      }
    }
  }
  return hmax;
}

// The one-sided (upwind) kinds -- external velocity arrays, LeVeque's
// deformation field, a constant velocity -- with two cells per thread, in
// the layout of stage_tile_pairs: thread (t, ty) of a TX/2 x TY block owns
// cells x0+2t and x0+2t+1 of row j0+ty and marches them along z, reading
// every ghost cell as stored.  Each cell takes one WENO5 side per axis, chosen
// by the sign of its velocity component (no face is shared between cells),
// so one barrier per plane suffices: plane k goes to buffer (k-kb)&1, and a
// thread writing that buffer again two planes on has passed the barrier of
// the plane between, which every reader of plane k has reached.  The pair
// reads its x stencils (cells x0+2t-4 .. x0+2t+5) as five and its y
// columns as seven 16-byte shared loads.  Per cell the arithmetic is that
// of stage_tile (weno_upwind_side and the same RHS and RK update), but for
// FP32 without the FP64 kink recomputation, where the two cells' sides of
// an axis are one packed FP32x2 evaluation (weno5_side2).
// BAND: the FP64 band form (out_alt written as well).
template <typename T, int KIND, bool K64, int TX, int TY, int TZ, bool BAND = false>
__device__ __forceinline__ void stage_tile_pairs_up(const StageParams<T>& p, int bx, int by,
                                                    int bz, T (*tile)[TY + 6][TX + 8]) {
  using T2 = typename Pair2<T>::type;
  // (no lane exchange: a row of TX/2 >= 4 threads of any width works)
  static_assert(TX % 2 == 0 && TX / 2 >= 4, "strip roles need four threads per row");
  static_assert(TY >= 3, "the y strips need three rows at each end");
  constexpr int NP = TX / 2;
  constexpr int PX = kPairPX;
  const int t = threadIdx.x, ty = threadIdx.y;
  const int x0 = p.fb.lo[0] + bx * TX, j0 = p.fb.lo[1] + by * TY;
  const int c0 = 2 * t;
  const int i0 = x0 + c0, i1 = i0 + 1;
  const int j = j0 + ty;
  const int kb = p.fb.lo[2] + bz * TZ;
  const int ke = min(kb + TZ - 1, p.fb.hi[2]);
  const int hi0 = p.fb.hi[0], hi1 = p.fb.hi[1];
  const bool rowin = j <= hi1;
  const bool act0 = rowin && i0 <= hi0, act1 = rowin && i1 <= hi0;
  const bool halo0 = !act0 && i0 <= hi0 + 3 && j <= hi1 + 3 && !(i0 > hi0 && j > hi1);
  const bool halo1 = !act1 && i1 <= hi0 + 3 && j <= hi1 + 3 && !(i1 > hi0 && j > hi1);
  const long sy = p.gb.sy(), sz = p.gb.sz();
  const long base0 = -((long)p.gb.lo[0] + sy * p.gb.lo[1] + sz * p.gb.lo[2]);
  const T dt = p.dt_dev ? (T)(*p.dt_dev) : (T)p.dt;
  const T ztol = stage_zero_tol<T>();

  // side strips and halo roles as in stage_tile_pairs
  int hxa = 0, hxb = 0;
  bool has_a = false, has_b = false;
  if (rowin) {
    if (t == 0) { hxa = x0 - 3; hxb = x0 - 2; has_a = has_b = true; }
    else if (t == 1) { hxa = x0 - 1; has_a = true; }
    else if (t == NP - 1) {
      hxa = x0 + TX; hxb = x0 + TX + 1;
      has_a = hxa <= hi0 + 3; has_b = hxb <= hi0 + 3;
    } else if (t == NP - 2) { hxa = x0 + TX + 2; has_a = hxa <= hi0 + 3; }
  }
  const int cola = hxa - x0 + PX, colb = hxb - x0 + PX;
  const int hj = ty < 3 ? j0 - 3 + ty : j + 3;
  const bool has_hy = (ty < 3) || (ty >= TY - 3 && rowin);
  const bool hy0 = has_hy && i0 <= hi0, hy1 = has_hy && i1 <= hi0;
  const int trow = ty < 3 ? ty : ty + 6;

  const T* P0 = p.phi_s + base0;
  const int isy = (int)sy, isz = (int)sz;
  auto ld = [&](int a, int b, int c) -> T { return __ldg(P0 + (a + isy * b + isz * c)); };
  T n0 = T(0), n1 = T(0), na = T(0), nb = T(0), ny0 = T(0), ny1 = T(0);
  auto prefetch = [&](int k) {
    if (act0) n0 = ld(i0, j, k + 3);
    else if (halo0) n0 = ld(i0, j, k);
    if (act1) n1 = ld(i1, j, k + 3);
    else if (halo1) n1 = ld(i1, j, k);
    if (has_a) na = ld(hxa, j, k);
    if (has_b) nb = ld(hxb, j, k);
    if (hy0) ny0 = ld(i0, hj, k);
    if (hy1) ny1 = ld(i1, hj, k);
  };

  T w0[7] = {}, w1[7] = {};
  if (act0) {
#pragma unroll
    for (int m = 0; m < 6; m++) w0[m + 1] = ld(i0, j, kb - 3 + m);
  }
  if (act1) {
#pragma unroll
    for (int m = 0; m < 6; m++) w1[m + 1] = ld(i1, j, kb - 3 + m);
  }
  prefetch(kb);
  for (int k = kb; k <= ke; ++k) {
    const int buf = (k - kb) & 1;
    T v0 = n0, v1 = n1;
    if (act0) {
#pragma unroll
      for (int m = 0; m < 6; m++) w0[m] = w0[m + 1];
      w0[6] = n0;
      v0 = w0[3];
    }
    if (act1) {
#pragma unroll
      for (int m = 0; m < 6; m++) w1[m] = w1[m + 1];
      w1[6] = n1;
      v1 = w1[3];
    }
    *reinterpret_cast<T2*>(&tile[buf][ty + 3][c0 + PX]) = T2{v0, v1};
    if (has_a) tile[buf][ty + 3][cola] = na;
    if (has_b) tile[buf][ty + 3][colb] = nb;
    if (hy0 || hy1) *reinterpret_cast<T2*>(&tile[buf][trow][c0 + PX]) = T2{ny0, ny1};
    __syncthreads();
    if (k < ke) prefetch(k + 1);
    if (!act0) continue;
    const long o0 = base0 + (i0 + isy * j + isz * k);
    // velocities and the RK input of both cells, loaded before the stencils
    T a[2][3] = {}, uc[2] = {};
#pragma unroll
    for (int c = 0; c < 2; c++) {
      if (c == 1 && !act1) break;
      const long o = o0 + c;
      if (KIND == kStageAdvect) {
        a[c][0] = __ldg(p.aux0 + o); a[c][1] = __ldg(p.aux1 + o); a[c][2] = __ldg(p.aux2 + o);
      } else if (KIND == kStageDeformation) {
        const int nx = p.fb.hi[0] - p.fb.lo[0] + 1, ny = p.fb.hi[1] - p.fb.lo[1] + 1,
                  nz = p.fb.hi[2] - p.fb.lo[2] + 1;
        const double* tx_ = p.defo_tab + p.defo_off[0] + (i0 + c - p.fb.lo[0]);
        const double* ty_ = p.defo_tab + p.defo_off[1] + (j - p.fb.lo[1]);
        const double* tz_ = p.defo_tab + p.defo_off[2] + (k - p.fb.lo[2]);
        DeformSines sn;
        sn.sx = __ldg(tx_); sn.s2x = __ldg(tx_ + nx);
        sn.sy = __ldg(ty_); sn.s2y = __ldg(ty_ + ny);
        sn.sz = __ldg(tz_); sn.s2z = __ldg(tz_ + nz);
        deformation_velocity(sn, __ldg(p.g_dev), a[c][0], a[c][1], a[c][2]);
      } else {
        a[c][0] = p.vel_const[0]; a[c][1] = p.vel_const[1]; a[c][2] = p.vel_const[2];
      }
      if (p.rk_kind != 1) uc[c] = __ldg(p.phi_n + o);
    }
    // one axis at a time for both cells, so that only one axis's stencils
    // are live: x from tile columns c0 .. c0+9 (phi(x0+2t-4 .. x0+2t+5)),
    // y from rows j-3 .. j+3 of the pair's two columns, z from the windows
    const bool kink64 = K64;
    T g[2][3] = {};
    // one axis for both cells: scalar sides, or (FP32 without the FP64 kink
    // recomputation) both cells' sides in one packed evaluation, each lane
    // with the differences of its own window in its own side's order
    auto axis = [&](int d, const T* wa, const T* wb) {
      const bool up0 = !(fabsT(a[0][d]) < ztol), up1 = act1 && !(fabsT(a[1][d]) < ztol);
      if constexpr (sizeof(T) == 4 && !K64) {
        const bool pl0 = !(a[0][d] > T(0)), pl1 = !(a[1][d] > T(0));
        float2 D[5];
#pragma unroll
        for (int m = 0; m < 5; m++)
          D[m] = make_float2(pl0 ? wa[6 - m] - wa[5 - m] : wa[m + 1] - wa[m],
                             pl1 ? wb[6 - m] - wb[5 - m] : wb[m + 1] - wb[m]);
        const float2 r = weno5_side2(D, p.inv[d]);
        if (up0) g[0][d] = r.x;
        if (up1) g[1][d] = r.y;
      } else {
        if (up0) g[0][d] = weno_upwind_side<T, true>(wa, p.inv[d], !(a[0][d] > T(0)), kink64);
        if (up1) g[1][d] = weno_upwind_side<T, true>(wb, p.inv[d], !(a[1][d] > T(0)), kink64);
      }
    };
    {
      T q[10];
#pragma unroll
      for (int m = 0; m < 5; m++) {
        const T2 v = *reinterpret_cast<const T2*>(&tile[buf][ty + 3][c0 + 2 * m]);
        q[2 * m] = v.x;
        q[2 * m + 1] = v.y;
      }
      axis(0, q + 1, q + 2);
    }
    {
      T ya[7], yb[7];
#pragma unroll
      for (int m = 0; m < 7; m++) {
        const T2 v = *reinterpret_cast<const T2*>(&tile[buf][ty + m][c0 + PX]);
        ya[m] = v.x;
        yb[m] = v.y;
      }
      axis(1, ya, yb);
    }
    axis(2, w0, w1);
#pragma unroll
    for (int c = 0; c < 2; c++) {
      if (c == 1 && !act1) break;
      const T L = T(0) - (a[c][0] * g[c][0] + a[c][1] * g[c][1] + a[c][2] * g[c][2]);
      const T v = stage_out(p, o0 + c, uc[c], c ? w1[3] : w0[3], L, dt);
      p.out[o0 + c] = v;
      if constexpr (BAND) store_alt(p.out_alt, o0 + c, v);
    }
  }
}

template <typename T, int KIND, bool FAST, int TX>
struct UseFaces {
  static constexpr bool value =
      (FAST || sizeof(T) == 4) && TX == 32 &&
      (KIND == kStageNormal || KIND == kStageReinit || KIND == kStageNormalRhs);
};
// the one-sided kinds of stage_tile_pairs_up
template <typename T, int KIND, bool FAST, int TX>
struct UsePairsUp {
  static constexpr bool value =
      (FAST || sizeof(T) == 4) && TX == 32 &&
      (KIND == kStageAdvect || KIND == kStageDeformation || KIND == kStageAdvectConst);
};

// kStageNormalRhs: the block's largest CFL speed into its partials slot,
// compared as the reference does ("if (h > m) m = h"); NT threads per block
template <int KIND, int NT, typename P>
__device__ __forceinline__ void block_max_partial(const P& p, double hmax) {
  if (KIND != kStageNormalRhs) return;
  __shared__ double red[NT / 32];
  double m = hmax;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double o2 = __shfl_xor_sync(0xffffffffu, m, off);
    m = (o2 > m) ? o2 : m;
  }
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) red[wid] = m;
  __syncthreads();
  if (wid == 0) {
    m = (lane < NT / 32) ? red[lane] : -1.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double o2 = __shfl_xor_sync(0xffffffffu, m, off);
      m = (o2 > m) ? o2 : m;
    }
    if (lane == 0)
      p.partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = m;
  }
}

// blocks per SM the register allocation must allow (default: 24 warps; with
// the 80 registers this leaves, the config-2 FP64 and FP32 stages run 6-7 %
// faster than with 16 warps at 128 registers)
#ifndef LSMGPU_STAGE_MIN_BLOCKS
#define LSMGPU_STAGE_MIN_BLOCKS (768 / (TX * TY))
#endif

template <typename T, int KIND, bool FAST, int TX, int TY, int TZ>
__global__ void __launch_bounds__(TX * TY, LSMGPU_STAGE_MIN_BLOCKS)
k_stage(StageParams<T> p) {
  __shared__ T tile[2][TY + 6][TX + 6];
  double hmax;
  if constexpr (UseFaces<T, KIND, FAST, TX>::value) {
    __shared__ T fy[TY][TX];
    __shared__ T fx[TY];
    hmax = stage_tile_faces<T, KIND, TX, TY, TZ>(p, (int)blockIdx.x, (int)blockIdx.y,
                                                 (int)blockIdx.z, tile, fy, fx);
  } else {
    hmax = stage_tile<T, KIND, FAST, TX, TY, TZ>(p, (int)blockIdx.x, (int)blockIdx.y,
                                                 (int)blockIdx.z, tile);
  }
  block_max_partial<KIND, TX * TY>(p, hmax);
}

// blocks per SM the register allocation of the pair kernel must allow
#ifndef LSMGPU_PAIR_MIN_BLOCKS
#define LSMGPU_PAIR_MIN_BLOCKS 4
#endif

// The face-shared two-sided kinds, two cells per thread (stage_tile_pairs):
// a block of TX/2 x TY threads covers the same TX x TY x TZ tile as k_stage.
// Every ghost cell the stencils reach is read as stored.
template <typename T, int KIND, bool K64, int TX, int TY, int TZ>
__global__ void __launch_bounds__(TX / 2 * TY, LSMGPU_PAIR_MIN_BLOCKS)
k_stage_pairs(StageParams<T> p) {
  __shared__ __align__(16) T tile[2][TY + 6][TX + 8];
  __shared__ __align__(16) T fy[TY][TX];
  __shared__ T fx[TY];
  const double hmax = stage_tile_pairs<T, KIND, K64, TX, TY, TZ>(
      p, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, tile, fy, fx);
  block_max_partial<KIND, TX / 2 * TY>(p, hmax);
}

// The one-sided kinds, two cells per thread (stage_tile_pairs_up); every
// ghost cell the stencils reach is read as stored.  BAND: the FP64 band form
// (the tiles whose tile_fp64 flag is tile_want, out_alt written as well).
template <typename T, int KIND, bool K64, int TX, int TY, int TZ, bool BAND = false>
__global__ void __launch_bounds__(TX / 2 * TY, LSMGPU_PAIR_MIN_BLOCKS)
k_stage_pairs_up(StageParams<T> p) {
  __shared__ __align__(16) T tile[2][TY + 6][TX + 8];
  if constexpr (BAND) {
    if (p.tile_fp64[blockIdx.x + gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z)] !=
        p.tile_want)
      return;
  }
  stage_tile_pairs_up<T, KIND, K64, TX, TY, TZ, BAND>(p, (int)blockIdx.x, (int)blockIdx.y,
                                                     (int)blockIdx.z, tile);
}

// The face ghost cells of phi that the stencils of fill-box cells in planes
// [k0, k1] read, written as stored values: beyond face f of the domain box
// (bits of bc_mask as in fetch_bc) the 3 layers over the domain's
// cross-section, from the same expressions as fetch_bc (linear: e0 +
// (e0 - e1) dist; copy: e0; periodic: the cell one period in).  x and y
// faces over planes [k0, k1]; the z faces when stencils of those planes
// reach them.  Each value depends on cells of the domain box only (no edge
// or corner ghost is read or written), so the threads are independent; the
// launcher requires at least 3 domain cells along every axis with a bit set.
// The grid is about one wave, each thread with the loads of several cells
// in flight (a version that looped a block over a plane's items waited on
// each iteration's loads in turn): per group of kGhostPlanes planes from
// k0, face_ghost_xy_blocks(nx, ny) blocks -- the x ghosts (the 6 cells of a
// row's two ends together, item 6 j + side * 3 + layer), then the y ghosts
// (6 rows along x, item nx (side * 3 + layer) + i), the same cell of each
// plane of the group per thread -- and after them zchunks blocks for each
// of the 6 z ghost planes.
template <typename T>
__device__ __forceinline__ T face_ghost_value(const Grid3<T>& g, const FillBox& dom,
                                              unsigned m, int face, int dist, T* cell) {
  const int d = face >> 1;
  const bool hi = face & 1;
  const long st = g.stride(d);
  if (m & (1u << (16 + face))) return *(cell + (hi ? -st : st) * dom.n(d));
  const T* e = cell + (hi ? -st : st) * dist;   // the domain's cell on the face
  const T e0 = *e;
  if (m & (1u << (8 + face))) return e0;
  const T e1 = *(e + (hi ? -st : st));
  const T slope = e0 - e1;
  return e0 + slope * (T)dist;
}

constexpr int kFaceGhostThreads = 256;

// item(r, v) for r = first, first + stride, ... below end, U items at a time
// with the loads of all U issued before any of their stores (the ghost
// fills are bound by load latency).  item returns the cell to write
// (nullptr: none) and sets v.
template <int U, typename T, typename F>
__device__ __forceinline__ void ghost_items(int first, int end, int stride, F item) {
  for (int r0 = first; r0 < end; r0 += U * stride) {
    T v[U];
    T* d[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int r = r0 + u * stride;
      d[u] = r < end ? item(r, v[u]) : nullptr;
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (d[u]) *d[u] = v[u];
  }
}

// planes per block of the x and y ghosts (one cell of each plane per thread,
// all their loads issued before the stores)
constexpr int kGhostPlanes = 4;

// blocks per group of kGhostPlanes planes for the x and y ghosts
__host__ __device__ inline int face_ghost_xy_blocks(int nx, int ny, int* bx = nullptr) {
  const int x = (6 * ny + kFaceGhostThreads - 1) / kFaceGhostThreads;
  if (bx) *bx = x;
  return x + (6 * nx + kFaceGhostThreads - 1) / kFaceGhostThreads;
}

template <typename T>
__global__ void __launch_bounds__(kFaceGhostThreads)
k_face_ghosts(T* phi, Box gb, FillBox dom, unsigned m, int k0, int k1, int zchunks) {
  const int nx = dom.n(0), ny = dom.n(1);
  const int ngroups = (k1 - k0 + kGhostPlanes) / kGhostPlanes;
  int bx;
  const int bxy = face_ghost_xy_blocks(nx, ny, &bx);
  const Grid3<T> g = make_grid(phi, gb);
  const unsigned any_face[6] = {m & 0x10101u, m & 0x20202u, m & 0x40404u,
                                m & 0x80808u, m & 0x101010u, m & 0x202020u};
  const int b = (int)blockIdx.x;
  if (b < ngroups * bxy) {
    const int ka = k0 + (b / bxy) * kGhostPlanes, sub = b % bxy;
    int face, dist, i, j;
    if (sub < bx) {
      const int q = sub * kFaceGhostThreads + (int)threadIdx.x;
      if (q >= 6 * ny) return;
      const int r = q % 6;
      j = dom.lo[1] + q / 6;
      face = r / 3;
      dist = r % 3 + 1;
      i = face ? dom.hi[0] + dist : dom.lo[0] - dist;
    } else {
      const int q = (sub - bx) * kFaceGhostThreads + (int)threadIdx.x;
      if (q >= 6 * nx) return;
      const int r = q / nx;
      i = dom.lo[0] + (q - r * nx);
      face = 2 + r / 3;
      dist = r % 3 + 1;
      j = face == 3 ? dom.hi[1] + dist : dom.lo[1] - dist;
    }
    if (!any_face[face]) return;
    T* const cell = g.ptr(i, j, ka);
    T v[kGhostPlanes];
#pragma unroll
    for (int u = 0; u < kGhostPlanes; u++)
      if (ka + u <= k1) v[u] = face_ghost_value(g, dom, m, face, dist, cell + u * g.sz);
#pragma unroll
    for (int u = 0; u < kGhostPlanes; u++)
      if (ka + u <= k1) cell[u * g.sz] = v[u];
    return;
  }
  // z ghost planes: plane zp = side * 3 + layer, chunk of its nx * ny cells
  const int zb = b - ngroups * bxy;
  const int zp = zb / zchunks, chunk = zb % zchunks;
  const int face = 4 + zp / 3, dist = zp % 3 + 1;
  if (!any_face[face]) return;
  if (face == 4 ? k0 - 3 >= dom.lo[2] : k1 + 3 <= dom.hi[2]) return;   // not reached
  const int k = face == 5 ? dom.hi[2] + dist : dom.lo[2] - dist;
  const int cells = nx * ny, per = (cells + zchunks - 1) / zchunks;
  const int end = min(cells, (chunk + 1) * per);
  ghost_items<4, T>(chunk * per + (int)threadIdx.x, end, kFaceGhostThreads,
                    [&](int q, T& v) -> T* {
                      const int i = dom.lo[0] + q % nx, j = dom.lo[1] + q / nx;
                      T* const cell = g.ptr(i, j, k);
                      v = face_ghost_value(g, dom, m, face, dist, cell);
                      return cell;
                    });
}

}  // namespace lsmgpu
