// adjoint.cu -- discrete adjoint of WENO5 upwind advection + TVD-RK3.
//
// Forward model (FP64): phi_t + V(x; theta).grad phi = 0 on a uniform grid
// with linear-extrapolation ghost values, V a trilinear B-spline on an
// m^3 control lattice spanning the domain, upwind HJ-WENO5 derivatives
// (LSM3D_UPWIND_HJ_WENO5, lsm_spatial_derivatives3d.f.in:2628-3000), the
// advection RHS (lsm_level_set_evolution3d.f.in:84-87) and TVD-RK3 stages
// (lsm_tvd_runge_kutta3d.f), dt frozen.  Loss
//   J = sum_cells (H(phi_T) - H(phi_target))^2 dx dy dz
// with H = LSM_HEAVISIDE(., eps) (lsm_calculus_toolbox.h:41-45).
//
// The reverse sweep is the exact transpose of the discrete forward map with
// the non-smooth choices frozen as the forward pass made them: the upwind
// side (sign of V at the cell), the zero-velocity cut, and the argmax inside
// the WENO eps.  For one RK3 step phi -> phi1 -> phi2 -> phi' and the adjoint
// lam = dJ/dphi':
//   mu3 = 2/3 dt lam;          lam2 = 2/3 lam + J(phi2)^T mu3
//   mu2 = 1/4 dt lam2;         lam1 = 1/4 lam2 + J(phi1)^T mu2
//   mu1 = dt lam1;             dJ/dphi = 1/3 lam + 3/4 lam2 + lam1 + J(phi)^T mu1
// where J(u)^T mu is the transposed Jacobian of L(u) = -V.grad_up(u), and the
// velocity adjoint accumulates A_d += -mu D_d(u) per cell, projected onto the
// B-spline basis once at the end.  States inside a checkpoint segment are
// recomputed from the segment's first state (sqrt(N) checkpointing).
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "capi_common.h"
#include "launch.h"
#include "stage.cuh"
#include "stage_launch.h"

using namespace lsmgpu;

namespace {

// tile of k_adjoint_stage: kTX x kTY cells per block, kTZ planes per block
// (build-time setting).  Short tiles balance the SMs: at 128^3 with two
// blocks per SM, 32-plane tiles make 256 blocks (108 SMs with two, 40 with
// one); 8-plane tiles make 1024 (about 7 per SM).  Measured reverse sweep of
// the 128^3 problem: 207.1 ms (32 planes), 201.9 (16), 200.8 (8).
#ifndef LSMGPU_ADJ_TZ
#define LSMGPU_ADJ_TZ 8
#endif
constexpr int kTX = 32, kTY = 8, kTZ = LSMGPU_ADJ_TZ;

// ---------------------------------------------------------------------------
// one-sided WENO5 value and its gradient with respect to v1..v5
//   D = sum w_k p_k,  w_k = a_k / sum a,  a_k = d_k / (S_k + eps)^2
//   dD/dv = sum w_k dp_k + sum b_k (dS_k + deps),
//   b_k = -2 w_k (p_k - D) / (S_k + eps)
// The weights use the single-reciprocal normalisation of the forward stage
// kernels (weno_fast.cuh): q_k = (S_k + eps) s with s a power of two,
// w_k = d_k prod_{j!=k} q_j^2 / sum_m (...), and the three 1/(S_k + eps)
// come from one more reciprocal, 1/q_k = s prod_{j!=k} q_j / (q_1 q_2 q_3).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void weno5_value_grad(const double v[5], double& D,
                                                 double g[5]) {
  const double a = 1.0 / 3.0, b = 7.0 / 6.0, c = 11.0 / 6.0, d = 1.0 / 6.0,
               e = 5.0 / 6.0;
  // eps: first maximum of v_j^2, as a chain of "if (x > m) m = x"
  int am = 0;
  double m = v[0] * v[0];
#pragma unroll
  for (int j = 1; j < 5; j++) {
    const double s = v[j] * v[j];
    if (s > m) { m = s; am = j; }
  }
  const double eps = 1e-6 * m + Consts<double>::tiny;
  const double p1 = a * v[0] - b * v[1] + c * v[2];
  const double p2 = -d * v[1] + e * v[2] + a * v[3];
  const double p3 = a * v[2] + e * v[3] - d * v[4];
  const double t1 = v[0] - 2 * v[1] + v[2], u1 = v[0] - 4 * v[1] + 3 * v[2];
  const double t2 = v[1] - 2 * v[2] + v[3], u2 = v[1] - v[3];
  const double t3 = v[2] - 2 * v[3] + v[4], u3 = 3 * v[2] - 4 * v[3] + v[4];
  const double S1 = 13.0 / 12.0 * t1 * t1 + 0.25 * u1 * u1;
  const double S2 = 13.0 / 12.0 * t2 * t2 + 0.25 * u2 * u2;
  const double S3 = 13.0 / 12.0 * t3 * t3 + 0.25 * u3 * u3;
  const double sc = inv_pow2_of(eps);
  const double es = eps * sc;
  const double q1 = S1 * sc + es, q2 = S2 * sc + es, q3 = S3 * sc + es;
  const double Q1 = q1 * q1, Q2 = q2 * q2, Q3 = q3 * q3;
  const double n1 = 0.1 * (Q2 * Q3), n2 = 0.6 * (Q1 * Q3), n3 = 0.3 * (Q1 * Q2);
  const double rn = rcp_nr(n1 + n2 + n3);
  const double w1 = n1 * rn, w2 = n2 * rn, w3 = n3 * rn;
  D = w1 * p1 + w2 * p2 + w3 * p3;
  const double rq = rcp_nr(q1 * q2 * q3) * sc;   // 1 / ((S1+eps)(S2+eps)(S3+eps)) / s^2
  const double b1 = -2.0 * w1 * (p1 - D) * (q2 * q3 * rq);
  const double b2 = -2.0 * w2 * (p2 - D) * (q1 * q3 * rq);
  const double b3 = -2.0 * w3 * (p3 - D) * (q1 * q2 * rq);
  const double k1 = 13.0 / 6.0 * t1, l1 = 0.5 * u1;
  const double k2 = 13.0 / 6.0 * t2, l2 = 0.5 * u2;
  const double k3 = 13.0 / 6.0 * t3, l3 = 0.5 * u3;
  // dp_k and dS_k, column by column
  g[0] = w1 * a + b1 * (k1 + l1);
  g[1] = -w1 * b - w2 * d + b1 * (-2 * k1 - 4 * l1) + b2 * (k2 + l2);
  g[2] = w1 * c + w2 * e + w3 * a + b1 * (k1 + 3 * l1) + b2 * (-2 * k2) +
         b3 * (k3 + 3 * l3);
  g[3] = w2 * a + w3 * e + b2 * (k2 - l2) + b3 * (-2 * k3 - 4 * l3);
  g[4] = -w3 * d + b3 * (k3 + l3);
  const double bs = (b1 + b2 + b3) * 2e-6 * v[am];
  g[am] += bs;
}

// Upwind derivative at the centre of w[0..6] = u(c-3..c+3) and its partials
// dD/dw[0..6]; minus side when vel > 0 (v = differences of w[0..5]), plus
// side otherwise (v = differences of w[6..1]); zero below the zero tolerance.
__device__ __forceinline__ double upwind_grad(const double* w, double inv,
                                              double vel, double dw[7]) {
#pragma unroll
  for (int m = 0; m < 7; m++) dw[m] = 0.0;
  if (fabs(vel) < Consts<double>::zero_tol) return 0.0;
  double v[5], g[5], D;
  if (vel > 0) {
#pragma unroll
    for (int j = 0; j < 5; j++) v[j] = (w[j + 1] - w[j]) * inv;
    weno5_value_grad(v, D, g);
    // v_j = (w_{j+1} - w_j) inv (0-based j)
#pragma unroll
    for (int j = 0; j < 5; j++) {
      dw[j + 1] += g[j] * inv;
      dw[j] -= g[j] * inv;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 5; j++) v[j] = (w[6 - j] - w[5 - j]) * inv;
    weno5_value_grad(v, D, g);
#pragma unroll
    for (int j = 0; j < 5; j++) {
      dw[6 - j] += g[j] * inv;
      dw[5 - j] -= g[j] * inv;
    }
  }
  return D;
}

struct AdjParams {
  const double* phi;      // stage input state u (stencil)
  const double* vel[3];   // velocity arrays
  const double* src_a;    // mu = coef * (ca * src_a + cb * src_b)
  double* src_b;          // zeroed after reading when zero_b (a consumed T)
  bool zero_b;
  double ca, cb, coef;
  double* src_out;        // optional: stores ca * src_a + cb * src_b
  double* T;              // += J(u)^T mu (atomic, zeroed by the caller)
  double* A[3];           // += -mu D_d(u)
  Box gb;
  FillBox fb;             // the domain (fill box = domain box)
  double inv[3];
};

// index of (i,j,k) in a gb array
__device__ __forceinline__ long aix(const Box& gb, int i, int j, int k) {
  return (long)(i - gb.lo[0]) + gb.sy() * (j - gb.lo[1]) + gb.sz() * (k - gb.lo[2]);
}

// Add val to T at a target that may lie one axis outside the domain: a ghost
// target is folded back through the linear extrapolation that produced it,
// g = e0 + (e0 - e1) dist, i.e. (1+dist) val to e0 and -dist val to e1.
__device__ __forceinline__ void add_target(const AdjParams& p, int i, int j, int k,
                                           double val) {
  const FillBox& f = p.fb;
  int c[3] = {i, j, k};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (c[d] < f.lo[d] || c[d] > f.hi[d]) {
      const bool lo = c[d] < f.lo[d];
      const int dist = lo ? f.lo[d] - c[d] : c[d] - f.hi[d];
      int e0[3] = {c[0], c[1], c[2]}, e1[3] = {c[0], c[1], c[2]};
      e0[d] = lo ? f.lo[d] : f.hi[d];
      e1[d] = lo ? f.lo[d] + 1 : f.hi[d] - 1;
      atomicAdd(p.T + aix(p.gb, e0[0], e0[1], e0[2]), (1.0 + dist) * val);
      atomicAdd(p.T + aix(p.gb, e1[0], e1[1], e1[2]), -(double)dist * val);
      return;
    }
  }
  atomicAdd(p.T + aix(p.gb, i, j, k), val);
}

// linear-extrapolation value of u at a point at most one axis outside
__device__ __forceinline__ double load_bc(const AdjParams& p, int i, int j, int k) {
  const FillBox& f = p.fb;
  int c[3] = {i, j, k};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (c[d] < f.lo[d] || c[d] > f.hi[d]) {
      const bool lo = c[d] < f.lo[d];
      const int dist = lo ? f.lo[d] - c[d] : c[d] - f.hi[d];
      int e0[3] = {c[0], c[1], c[2]}, e1[3] = {c[0], c[1], c[2]};
      e0[d] = lo ? f.lo[d] : f.hi[d];
      e1[d] = lo ? f.lo[d] + 1 : f.hi[d] - 1;
      const double a = __ldg(p.phi + aix(p.gb, e0[0], e0[1], e0[2]));
      const double b = __ldg(p.phi + aix(p.gb, e1[0], e1[1], e1[2]));
      return a + (a - b) * (double)dist;
    }
  }
  return __ldg(p.phi + aix(p.gb, i, j, k));
}

// Transposed Jacobian of the upwind advection RHS.  Every cell c owns the
// partials -V_d(c) mu(c) dD_d(c)/du(p) of its stencil points p.  The z
// contributions go through a 7-plane register ring along the march; the x/y
// contributions of a plane are written to shared memory (seven per axis per
// cell) and gathered by the thread of each target cell, without atomics.
// Each finished plane of the ring and the contributions to the neighbouring
// tiles (3-cell strips) are added to T with atomics.
__global__ void __launch_bounds__(kTX * kTY, 2)
k_adjoint_stage(AdjParams p) {
  __shared__ double tile[kTY + 6][kTX + 6];
  __shared__ double Cx[7][kTY][kTX];
  __shared__ double Cy[7][kTY][kTX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = p.fb.lo[0] + (int)blockIdx.x * kTX + tx;
  const int j = p.fb.lo[1] + (int)blockIdx.y * kTY + ty;
  const int kb = p.fb.lo[2] + (int)blockIdx.z * kTZ;
  const int ke = min(kb + kTZ - 1, p.fb.hi[2]);
  const bool act = i <= p.fb.hi[0] && j <= p.fb.hi[1];
  const int hi0 = p.fb.hi[0], hi1 = p.fb.hi[1];
  const bool ctr_halo = !act && i <= hi0 + 3 && j <= hi1 + 3 && !(i > hi0 && j > hi1);
  const int hx = (tx < 3) ? (i - 3) : (i + 3);
  const bool has_hx = (j <= hi1) && ((tx < 3) || (tx >= kTX - 3 && i <= hi0));
  const int hj = (ty < 3) ? (j - 3) : (j + 3);
  const bool has_hy = (i <= hi0) && ((ty < 3) || (ty >= kTY - 3 && j <= hi1));
  const int tcol = (tx < 3) ? tx : tx + 6;
  const int trow = (ty < 3) ? ty : ty + 6;
  // tiles whose stencils stay inside the domain load without boundary tests
  const int x0 = p.fb.lo[0] + (int)blockIdx.x * kTX, y0 = p.fb.lo[1] + (int)blockIdx.y * kTY;
  const bool inside = x0 - 3 >= p.fb.lo[0] && min(x0 + kTX - 1, hi0) + 3 <= hi0 &&
                      y0 - 3 >= p.fb.lo[1] && min(y0 + kTY - 1, hi1) + 3 <= hi1 &&
                      kb - 3 >= p.fb.lo[2] && ke + 3 <= p.fb.hi[2];
  auto ld = [&](int a, int b, int c) -> double {
    return inside ? __ldg(p.phi + aix(p.gb, a, b, c)) : load_bc(p, a, b, c);
  };

  // registers of the next plane (loaded while the current one is worked):
  // the new top of the z window or the own cell (halo threads), the strip
  // cells, and the own cell's velocity and adjoint sources
  double nx_c = 0.0, nx_hx = 0.0, nx_hy = 0.0, nv0 = 0.0, nv1 = 0.0, nv2 = 0.0,
         nsa = 0.0, nsb = 0.0;
  auto prefetch = [&](int k) {
    if (act) {
      nx_c = ld(i, j, k + 3);
      const long o = aix(p.gb, i, j, k);
      nv0 = __ldg(p.vel[0] + o);
      nv1 = __ldg(p.vel[1] + o);
      nv2 = __ldg(p.vel[2] + o);
      nsa = p.src_a[o];
      if (p.src_b) nsb = p.src_b[o];
    } else if (ctr_halo) {
      nx_c = ld(i, j, k);
    }
    if (has_hx) nx_hx = ld(hx, j, k);
    if (has_hy) nx_hy = ld(i, hj, k);
  };

  double w[7], ring[7];
#pragma unroll
  for (int m = 0; m < 7; m++) ring[m] = 0.0;
  if (act) {
#pragma unroll
    for (int m = 0; m < 6; m++) w[m + 1] = ld(i, j, kb - 3 + m);
  }
  prefetch(kb);
  for (int k = kb; k <= ke; ++k) {
    const double vx = nv0, vy = nv1, vz = nv2, sa = nsa, sb = nsb;
    if (act) {
#pragma unroll
      for (int m = 0; m < 6; m++) w[m] = w[m + 1];
      w[6] = nx_c;
      tile[ty + 3][tx + 3] = w[3];
    } else if (ctr_halo) {
      tile[ty + 3][tx + 3] = nx_c;
    }
    if (has_hx) tile[ty + 3][tcol] = nx_hx;
    if (has_hy) tile[trow][tx + 3] = nx_hy;
    __syncthreads();
    if (k < ke) prefetch(k + 1);
    if (act) {
      const long o = aix(p.gb, i, j, k);
      const double a0 = p.A[0][o], a1 = p.A[1][o], a2 = p.A[2][o];
      double src = p.ca * sa;
      if (p.src_b) {
        src += p.cb * sb;
        if (p.zero_b) p.src_b[o] = 0.0;
      }
      if (p.src_out) p.src_out[o] = src;
      const double mu = p.coef * src;
      // one axis at a time: its seven partials are consumed before the next
      // axis is differentiated; targets outside the domain are folded back
      // at once, the others wait in shared memory for the gather
      double Dx, Dy, Dz;
      {
        double wx[7], d7[7];
#pragma unroll
        for (int m = 0; m < 7; m++) wx[m] = tile[ty + 3][tx + m];
        Dx = upwind_grad(wx, p.inv[0], vx, d7);
        const double sx = -vx * mu;
#pragma unroll
        for (int m = 0; m < 7; m++) {
          double c = sx * d7[m];
          const int ti = i + m - 3;
          if (ti < p.fb.lo[0] || ti > hi0) {
            if (c != 0.0) add_target(p, ti, j, k, c);
            c = 0.0;
          }
          Cx[m][ty][tx] = c;
        }
      }
      {
        double wy[7], d7[7];
#pragma unroll
        for (int m = 0; m < 7; m++) wy[m] = tile[ty + m][tx + 3];
        Dy = upwind_grad(wy, p.inv[1], vy, d7);
        const double sy = -vy * mu;
#pragma unroll
        for (int m = 0; m < 7; m++) {
          double c = sy * d7[m];
          const int tj = j + m - 3;
          if (tj < p.fb.lo[1] || tj > hi1) {
            if (c != 0.0) add_target(p, i, tj, k, c);
            c = 0.0;
          }
          Cy[m][ty][tx] = c;
        }
      }
      {
        double d7[7];
        Dz = upwind_grad(w, p.inv[2], vz, d7);
        const double sz = -vz * mu;
#pragma unroll
        for (int m = 0; m < 7; m++) ring[m] += sz * d7[m];   // ring[m]: plane k+m-3
      }
      p.A[0][o] = a0 - mu * Dx;
      p.A[1][o] = a1 - mu * Dy;
      p.A[2][o] = a2 - mu * Dz;
    } else {
#pragma unroll
      for (int m = 0; m < 7; m++) {
        Cx[m][ty][tx] = 0.0;
        Cy[m][ty][tx] = 0.0;
      }
    }
    __syncthreads();
    // the x/y contributions of this plane to target column c / row r of the
    // tile (c, r may lie up to 3 outside it): sources s = c-3..c+3 in the tile
    auto gather_x = [&](int c) {
      double v = 0.0;
#pragma unroll
      for (int m = 0; m < 7; m++) {
        const int s = c + 3 - m;
        if (s >= 0 && s < kTX) v += Cx[m][ty][s];
      }
      return v;
    };
    auto gather_y = [&](int r) {
      double v = 0.0;
#pragma unroll
      for (int m = 0; m < 7; m++) {
        const int s = r + 3 - m;
        if (s >= 0 && s < kTY) v += Cy[m][s][tx];
      }
      return v;
    };
    if (act) {
      // own cell: plane k's in-plane sum joins the ring; the ring's oldest
      // plane (k-3) is complete and leaves through an atomic add
      ring[3] += gather_x(tx) + gather_y(ty);
      if (ring[0] != 0.0) add_target(p, i, j, k - 3, ring[0]);
#pragma unroll
      for (int m = 0; m < 6; m++) ring[m] = ring[m + 1];
      ring[6] = 0.0;
    }
    // contributions to the neighbouring tiles' cells next to this tile
    if (has_hx) {
      const double v = gather_x(tcol - 3);
      if (v != 0.0) add_target(p, hx, j, k, v);
    }
    if (has_hy) {
      const double v = gather_y(trow - 3);
      if (v != 0.0) add_target(p, i, hj, k, v);
    }
  }
  // planes ke-2 .. ke+3 still in the ring
  if (act) {
#pragma unroll
    for (int m = 0; m < 6; m++)
      if (ring[m] != 0.0) add_target(p, i, j, ke - 2 + m, ring[m]);
  }
}

// lam' = 1/3 lam + 3/4 lam2 + lam1 + T1 (pointwise, fill box); T1 is
// consumed (zeroed for the next step's accumulation)
__global__ void k_adj_combine(double* out, const double* lam, const double* lam2,
                              const double* lam1, double* T1, Box gb, FillBox fb) {
  const int i = fb.lo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = fb.lo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > fb.hi[0] || j > fb.hi[1]) return;
  for (int k = fb.lo[2] + blockIdx.z; k <= fb.hi[2]; k += gridDim.z) {
    const long o = aix(gb, i, j, k);
    out[o] = (1.0 / 3.0) * lam[o] + 0.75 * lam2[o] + lam1[o] + T1[o];
    T1[o] = 0.0;
  }
}

// trilinear B-spline (hat functions) on an m^3 lattice spanning [x0, x1]^3
struct Spline {
  int m;
  double lo[3], h[3];   // lattice origin and spacing per axis
};

__device__ __forceinline__ void hat(const Spline& s, int d, double x, int& a0,
                                    double& t) {
  double r = (x - s.lo[d]) / s.h[d];
  int a = (int)floor(r);
  if (a < 0) a = 0;
  if (a > s.m - 2) a = s.m - 2;
  a0 = a;
  t = r - a;
}

__global__ void k_spline_velocity(double* vx, double* vy, double* vz,
                                  const double* theta, Spline s, Box gb,
                                  FillBox fb, double x0, double y0, double z0,
                                  double dx, double dy, double dz) {
  const int i = fb.lo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = fb.lo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > fb.hi[0] || j > fb.hi[1]) return;
  int ax, ay;
  double tx, ty;
  hat(s, 0, x0 + (i + 0.5) * dx, ax, tx);
  hat(s, 1, y0 + (j + 0.5) * dy, ay, ty);
  const int m = s.m, m3 = m * m * m;
  for (int k = fb.lo[2] + blockIdx.z; k <= fb.hi[2]; k += gridDim.z) {
    int az;
    double tz;
    hat(s, 2, z0 + (k + 0.5) * dz, az, tz);
    double u[3] = {0, 0, 0};
    for (int c = 0; c < 2; c++)
      for (int b = 0; b < 2; b++)
        for (int a = 0; a < 2; a++) {
          const double wgt = (a ? tx : 1 - tx) * (b ? ty : 1 - ty) * (c ? tz : 1 - tz);
          const int q = (ax + a) + m * ((ay + b) + m * (az + c));
          u[0] += wgt * theta[q];
          u[1] += wgt * theta[m3 + q];
          u[2] += wgt * theta[2 * m3 + q];
        }
    const long o = aix(gb, i, j, k);
    vx[o] = u[0];
    vy[o] = u[1];
    vz[o] = u[2];
  }
}

// grad_theta[d][q] += sum_cells A_d(cell) * basis_q(cell); block-local sums
// in shared memory, one atomic per lattice coefficient per block
__global__ void k_spline_project(const double* A0, const double* A1, const double* A2,
                                 double* grad, Spline s, Box gb, FillBox fb,
                                 double x0, double y0, double z0, double dx,
                                 double dy, double dz) {
  extern __shared__ double sh[];
  const int m = s.m, m3 = m * m * m;
  for (int q = threadIdx.x; q < 3 * m3; q += blockDim.x) sh[q] = 0.0;
  __syncthreads();
  const long n = fb.count();
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const int i = fb.lo[0] + (int)(t % fb.n(0));
    const long r = t / fb.n(0);
    const int j = fb.lo[1] + (int)(r % fb.n(1));
    const int k = fb.lo[2] + (int)(r / fb.n(1));
    int ax, ay, az;
    double tx, ty, tz;
    hat(s, 0, x0 + (i + 0.5) * dx, ax, tx);
    hat(s, 1, y0 + (j + 0.5) * dy, ay, ty);
    hat(s, 2, z0 + (k + 0.5) * dz, az, tz);
    const long o = aix(gb, i, j, k);
    const double a[3] = {A0[o], A1[o], A2[o]};
    for (int c = 0; c < 2; c++)
      for (int b = 0; b < 2; b++)
        for (int e = 0; e < 2; e++) {
          const double wgt = (e ? tx : 1 - tx) * (b ? ty : 1 - ty) * (c ? tz : 1 - tz);
          const int q = (ax + e) + m * ((ay + b) + m * (az + c));
          atomicAdd(&sh[q], wgt * a[0]);
          atomicAdd(&sh[m3 + q], wgt * a[1]);
          atomicAdd(&sh[2 * m3 + q], wgt * a[2]);
        }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < 3 * m3; q += blockDim.x)
    if (sh[q] != 0.0) atomicAdd(grad + q, sh[q]);
}

// LSM_HEAVISIDE and its derivative
__device__ __forceinline__ double heav(double x, double eps) {
  if (x < -eps) return 0.0;
  if (x > eps) return 1.0;
  return 0.5 * (1 + x / eps + 1 / M_PI * sin(M_PI * x / eps));
}
__device__ __forceinline__ double dheav(double x, double eps) {
  if (x < -eps || x > eps) return 0.0;
  return 0.5 * (1.0 + cos(M_PI * x / eps)) / eps;
}

// per-block partial sums of the loss; lam = dJ/dphi_T when lam != nullptr
__global__ void k_loss(const double* phi, const double* target, double* lam,
                       double* partials, Box gb, FillBox fb, double eps, double vol) {
  __shared__ double red[8];
  double s = 0.0;
  const long n = fb.count();
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const int i = fb.lo[0] + (int)(t % fb.n(0));
    const long r = t / fb.n(0);
    const int j = fb.lo[1] + (int)(r % fb.n(1));
    const int k = fb.lo[2] + (int)(r / fb.n(1));
    const long o = aix(gb, i, j, k);
    const double d = heav(phi[o], eps) - heav(target[o], eps);
    s += d * d * vol;
    if (lam) lam[o] = 2.0 * d * dheav(phi[o], eps) * vol;
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += red[w];
    partials[blockIdx.x] = tot;
  }
}

constexpr int kLossBlocks = 296;

}  // namespace

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
struct lsmgpu_adjoint {
  Box gb;
  FillBox fb;
  double dx[3], x_lo[3];
  Spline spl;
  size_t bytes;
  double* vel[3] = {nullptr, nullptr, nullptr};
  double* theta = nullptr;
  double* grad_theta = nullptr;
  double* target = nullptr;
  double* phi = nullptr;        // working state
  double* s1 = nullptr;         // stage buffers
  double* s2 = nullptr;
  std::vector<double*> ckpt;    // checkpoint states
  // two sets of segment buffers: [set][0] the states u_s of a segment,
  // [set][1] and [set][2] their TVD-RK3 stage-1 and stage-2 states.  The
  // segment before the one being reversed is recomputed into the other set
  // on the auxiliary stream.
  std::vector<double*> segs[2][3];
  cudaStream_t aux = nullptr;
  cudaEvent_t ready[2] = {nullptr, nullptr};
  cudaEvent_t freed[2] = {nullptr, nullptr};
  cudaEvent_t start = nullptr;
  double* lam = nullptr;
  double* lam2 = nullptr;
  double* lam1 = nullptr;
  double* T = nullptr;          // two accumulation buffers of J^T mu; each is
  double* Tb = nullptr;         // zeroed by the kernel that consumes it
  double* A[3] = {nullptr, nullptr, nullptr};
  double* partials = nullptr;
  int nsteps = 0, every = 1;
  double dt = 0.0, eps = 0.0;
  float fwd_ms = 0.f, adj_ms = 0.f;
};

namespace {

double* dalloc(size_t bytes, bool& ok) {
  void* p = nullptr;
  if (ok && cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    ok = false;
    return nullptr;
  }
  if (ok) cudaMemset(p, 0, bytes);
  return (double*)p;
}

StageArgs fwd_args(lsmgpu_adjoint* h) {
  StageArgs a;
  memset(&a, 0, sizeof a);
  a.gb = h->gb;
  a.fb = h->fb;
  a.dom = h->fb;
  a.bc_mask = kBcLinear;
  for (int d = 0; d < 3; d++) a.inv[d] = 1.0 / h->dx[d];
  double m = std::max(std::max(h->dx[0], h->dx[1]), h->dx[2]);
  a.dx_sq = m * m;
  a.dt = h->dt;
  for (int d = 0; d < 3; d++) a.aux[d] = h->vel[d];
  return a;
}

cudaError_t fwd_stage(lsmgpu_adjoint* h, double* out, const double* in,
                      const double* base, int rk, cudaStream_t st) {
  StageArgs a = fwd_args(h);
  a.out = out;
  a.phi_s = in;
  a.phi_n = base;
  a.rk_kind = rk;
  return launch_stage_fast(kStageAdvect, 8, a, st);
}

// one forward TVD-RK3 step: out = step(in); out may equal in
cudaError_t fwd_step(lsmgpu_adjoint* h, double* out, const double* in, cudaStream_t st) {
  cudaError_t e;
  if ((e = fwd_stage(h, h->s1, in, in, 1, st))) return e;
  if ((e = fwd_stage(h, h->s2, h->s1, in, 32, st))) return e;
  return fwd_stage(h, out, h->s2, in, 33, st);
}

// T += J(u)^T mu with mu = coef (ca sa + cb sb); T must be zero on entry, sb
// (a consumed accumulation buffer, or null) is zeroed as it is read
cudaError_t adj_kernel(lsmgpu_adjoint* h, const double* u, const double* sa, double ca,
                       double* sb, double cb, double coef, double* sout, double* T,
                       cudaStream_t st) {
  AdjParams p;
  p.phi = u;
  for (int d = 0; d < 3; d++) {
    p.vel[d] = h->vel[d];
    p.A[d] = h->A[d];
    p.inv[d] = 1.0 / h->dx[d];
  }
  p.src_a = sa; p.ca = ca; p.src_b = sb; p.cb = cb; p.coef = coef; p.src_out = sout;
  p.zero_b = sb != nullptr;
  p.T = T;
  p.gb = h->gb;
  p.fb = h->fb;
  dim3 grid((h->fb.n(0) + kTX - 1) / kTX, (h->fb.n(1) + kTY - 1) / kTY,
            (h->fb.n(2) + kTZ - 1) / kTZ);
  k_adjoint_stage<<<grid, dim3(kTX, kTY), 0, st>>>(p);
  ++launch_counter();
  return cudaGetLastError();
}

// states u_s (s > first) of checkpoint segment c and the stage states of
// every step of it, recomputed from the segment's checkpoint into buffer set b
cudaError_t recompute_segment(lsmgpu_adjoint* h, int c, int b, cudaStream_t st) {
  const int s0 = c * h->every, s1 = std::min(s0 + h->every, h->nsteps);
  std::vector<double*>* set = h->segs[b];
  cudaError_t e;
  for (int s = s0; s < s1; s++) {
    const int q = s - s0;
    const double* u = q == 0 ? h->ckpt[c] : set[0][q];
    if ((e = fwd_stage(h, set[1][q], u, u, 1, st))) return e;
    if ((e = fwd_stage(h, set[2][q], set[1][q], u, 32, st))) return e;
    if (s + 1 < s1 && (e = fwd_stage(h, set[0][q + 1], set[2][q], u, 33, st))) return e;
  }
  return cudaSuccess;
}

// reverse one RK3 step whose input state is u and stage states s1, s2:
// lam <- dJ/du
cudaError_t adj_step(lsmgpu_adjoint* h, const double* u, const double* s1,
                     const double* s2, cudaStream_t st) {
  cudaError_t e;
  const double dt = h->dt;
  // stage 3: mu3 = 2/3 dt lam; T <- J(phi2)^T mu3
  if ((e = adj_kernel(h, s2, h->lam, 1.0, nullptr, 0.0, (2.0 / 3.0) * dt, nullptr, h->T,
                      st)))
    return e;
  // stage 2: lam2 = 2/3 lam + T3 (T consumed); mu2 = 1/4 dt lam2;
  // Tb <- J(phi1)^T mu2
  if ((e = adj_kernel(h, s1, h->lam, 2.0 / 3.0, h->T, 1.0, 0.25 * dt, h->lam2, h->Tb, st)))
    return e;
  // stage 1: lam1 = 1/4 lam2 + T2 (Tb consumed); mu1 = dt lam1;
  // T <- J(u)^T mu1
  if ((e = adj_kernel(h, u, h->lam2, 0.25, h->Tb, 1.0, dt, h->lam1, h->T, st))) return e;
  // lam <- 1/3 lam + 3/4 lam2 + lam1 + T1 (T consumed)
  dim3 blk(32, 4, 1), grid((h->fb.n(0) + 31) / 32, (h->fb.n(1) + 3) / 4,
                           h->fb.n(2) < 65535 ? h->fb.n(2) : 65535);
  k_adj_combine<<<grid, blk, 0, st>>>(h->lam, h->lam, h->lam2, h->lam1, h->T, h->gb, h->fb);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t loss_on_device(lsmgpu_adjoint* h, const double* phi, double* lam,
                           cudaStream_t st) {
  const double vol = h->dx[0] * h->dx[1] * h->dx[2];
  k_loss<<<kLossBlocks, 256, 0, st>>>(phi, h->target, lam, h->partials, h->gb, h->fb,
                                      h->eps, vol);
  ++launch_counter();
  return cudaGetLastError();
}

bool loss_to_host(lsmgpu_adjoint* h, double* loss, cudaStream_t st, const char* R) {
  double part[kLossBlocks];
  if (!cuda_ok(cudaMemcpyAsync(part, h->partials, sizeof part, cudaMemcpyDeviceToHost, st),
               R) ||
      !cuda_ok(cudaStreamSynchronize(st), R))
    return false;
  double s = 0.0;
  for (int b = 0; b < kLossBlocks; b++) s += part[b];
  *loss = s;
  return true;
}

// forward run from phi0 (h->ckpt[0] holds phi0 after set_fields), storing the
// checkpoints; the final state is left in h->phi
cudaError_t forward_run(lsmgpu_adjoint* h, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(h->phi, h->ckpt[0], h->bytes, cudaMemcpyDeviceToDevice, st);
  if (e) return e;
  for (int s = 0; s < h->nsteps; s++) {
    if (s % h->every == 0 && s > 0)
      if ((e = cudaMemcpyAsync(h->ckpt[s / h->every], h->phi, h->bytes,
                               cudaMemcpyDeviceToDevice, st)))
        return e;
    if ((e = fwd_step(h, h->phi, h->phi, st))) return e;
  }
  return cudaSuccess;
}

}  // namespace

extern "C" {

// Create an adjoint problem on an n^3 interior grid over [x_lo, x_lo + n*dx]
// with a trilinear B-spline velocity on an m^3 lattice spanning the domain.
int lsmgpu_adjoint_create(lsmgpu_adjoint** out, const int n[3], const double dx[3],
                          const double x_lo[3], int lattice, int nsteps,
                          int checkpoint_every) {
  const char* R = "lsmgpu_adjoint_create";
  clear_error();
  if (!out || !n || !dx || !x_lo) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  *out = nullptr;
  if (lattice < 2 || nsteps < 1 || checkpoint_every < 1 || n[0] < 4 || n[1] < 4 ||
      n[2] < 4) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": bad sizes");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  lsmgpu_adjoint* h = new lsmgpu_adjoint();
  for (int d = 0; d < 3; d++) {
    h->gb.lo[d] = -3;
    h->gb.n[d] = n[d] + 6;
    h->fb.lo[d] = 0;
    h->fb.hi[d] = n[d] - 1;
    h->dx[d] = dx[d];
    h->x_lo[d] = x_lo[d];
    h->spl.lo[d] = x_lo[d];
    h->spl.h[d] = n[d] * dx[d] / (lattice - 1);
  }
  h->spl.m = lattice;
  h->bytes = (size_t)h->gb.count() * sizeof(double);
  h->nsteps = nsteps;
  h->every = checkpoint_every;
  const int nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
  bool ok = true;
  for (int d = 0; d < 3; d++) {
    h->vel[d] = dalloc(h->bytes, ok);
    h->A[d] = dalloc(h->bytes, ok);
  }
  const size_t m3 = (size_t)lattice * lattice * lattice;
  h->theta = dalloc(3 * m3 * sizeof(double), ok);
  h->grad_theta = dalloc(3 * m3 * sizeof(double), ok);
  h->target = dalloc(h->bytes, ok);
  h->phi = dalloc(h->bytes, ok);
  h->s1 = dalloc(h->bytes, ok);
  h->s2 = dalloc(h->bytes, ok);
  h->lam = dalloc(h->bytes, ok);
  h->lam2 = dalloc(h->bytes, ok);
  h->lam1 = dalloc(h->bytes, ok);
  h->T = dalloc(h->bytes, ok);
  h->Tb = dalloc(h->bytes, ok);
  h->partials = dalloc(kLossBlocks * sizeof(double), ok);
  for (int c = 0; c < nck; c++) h->ckpt.push_back(dalloc(h->bytes, ok));
  for (int b = 0; b < 2; b++)
    for (int v = 0; v < 3; v++)
      for (int c = 0; c < checkpoint_every; c++) h->segs[b][v].push_back(dalloc(h->bytes, ok));
  ok = ok && cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking) == cudaSuccess;
  for (int b = 0; ok && b < 2; b++)
    ok = cudaEventCreateWithFlags(&h->ready[b], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&h->freed[b], cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&h->start, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    set_error(LSMGPU_ERR_ALLOC, std::string(R) + ": device allocation failed");
    lsmgpu_adjoint_destroy(h);
    return LSMGPU_ERR_ALLOC;
  }
  *out = h;
  return LSMGPU_SUCCESS;
}

int lsmgpu_adjoint_destroy(lsmgpu_adjoint* h) {
  if (!h) return LSMGPU_SUCCESS;
  double* ps[] = {h->vel[0], h->vel[1], h->vel[2], h->A[0], h->A[1], h->A[2],
                  h->theta, h->grad_theta, h->target, h->phi, h->s1, h->s2,
                  h->lam, h->lam2, h->lam1, h->T, h->Tb, h->partials};
  for (double* p : ps)
    if (p) cudaFree(p);
  for (double* p : h->ckpt)
    if (p) cudaFree(p);
  if (h->aux) cudaStreamSynchronize(h->aux);
  for (auto& set : h->segs)
    for (auto& v : set)
      for (double* p : v)
        if (p) cudaFree(p);
  for (cudaEvent_t ev : {h->ready[0], h->ready[1], h->freed[0], h->freed[1], h->start})
    if (ev) cudaEventDestroy(ev);
  if (h->aux) cudaStreamDestroy(h->aux);
  delete h;
  return LSMGPU_SUCCESS;
}

// B-spline coefficients theta[3][m][m][m] (x fastest; component-major) from
// the host; evaluates the velocity arrays
int lsmgpu_adjoint_set_theta(lsmgpu_adjoint* h, const double* theta) {
  const char* R = "lsmgpu_adjoint_set_theta";
  clear_error();
  if (!h || !theta) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  const size_t m3 = (size_t)h->spl.m * h->spl.m * h->spl.m;
  cudaStream_t st = cur_stream();
  if (!cuda_ok(cudaMemcpyAsync(h->theta, theta, 3 * m3 * sizeof(double),
                               cudaMemcpyHostToDevice, st),
               R))
    return LSMGPU_ERR_CUDA;
  dim3 blk(32, 4, 1), grid((h->fb.n(0) + 31) / 32, (h->fb.n(1) + 3) / 4,
                           h->fb.n(2) < 65535 ? h->fb.n(2) : 65535);
  k_spline_velocity<<<grid, blk, 0, st>>>(h->vel[0], h->vel[1], h->vel[2], h->theta,
                                          h->spl, h->gb, h->fb, h->x_lo[0], h->x_lo[1],
                                          h->x_lo[2], h->dx[0], h->dx[1], h->dx[2]);
  ++launch_counter();
  return cuda_ok(cudaGetLastError(), R) ? LSMGPU_SUCCESS : LSMGPU_ERR_CUDA;
}

// CFL dt of the current velocity (LSM3D_COMPUTE_STABLE_ADVECTION_DT)
int lsmgpu_adjoint_cfl_dt(lsmgpu_adjoint* h, double cfl, double* dt) {
  const char* R = "lsmgpu_adjoint_cfl_dt";
  clear_error();
  if (!h || !dt) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  cudaStream_t st = cur_stream();
  ReduceScratch scr(st, reduce_partials_needed(h->fb));
  if (!scr.ok()) return LSMGPU_ERR_ALLOC;
  const void* v[3] = {h->vel[0], h->vel[1], h->vel[2]};
  const double inv[3] = {1.0 / h->dx[0], 1.0 / h->dx[1], 1.0 / h->dx[2]};
  if (!cuda_ok(launch_stable_advection_dt(8, v, h->gb, h->fb, inv, cfl, scr.partials(),
                                          scr.result(), st),
               R))
    return LSMGPU_ERR_CUDA;
  if (!cuda_ok(cudaMemcpyAsync(dt, scr.result(), sizeof(double), cudaMemcpyDeviceToHost,
                               st),
               R) ||
      !cuda_ok(cudaStreamSynchronize(st), R))
    return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

int lsmgpu_adjoint_set_dt(lsmgpu_adjoint* h, double dt) {
  if (!h) return LSMGPU_ERR_NULL_POINTER;
  h->dt = dt;
  return LSMGPU_SUCCESS;
}

// phi0 and the target level set (host arrays over the ghost box) and the
// Heaviside width
int lsmgpu_adjoint_set_fields(lsmgpu_adjoint* h, const double* phi0,
                              const double* target, double eps) {
  const char* R = "lsmgpu_adjoint_set_fields";
  clear_error();
  if (!h || !phi0 || !target) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  h->eps = eps;
  cudaStream_t st = cur_stream();
  return cuda_ok(cudaMemcpyAsync(h->ckpt[0], phi0, h->bytes, cudaMemcpyHostToDevice, st),
                 R) &&
                 cuda_ok(cudaMemcpyAsync(h->target, target, h->bytes,
                                         cudaMemcpyHostToDevice, st),
                         R) &&
                 cuda_ok(cudaStreamSynchronize(st), R)
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}

// forward run and loss
int lsmgpu_adjoint_forward(lsmgpu_adjoint* h, double* loss) {
  const char* R = "lsmgpu_adjoint_forward";
  clear_error();
  if (!h || !loss) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  cudaStream_t st = cur_stream();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  bool ok = cuda_ok(forward_run(h, st), R) && cuda_ok(loss_on_device(h, h->phi, nullptr, st), R);
  cudaEventRecord(e1, st);
  ok = ok && loss_to_host(h, loss, st, R);
  if (ok) cudaEventElapsedTime(&h->fwd_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ok ? LSMGPU_SUCCESS : lsmgpu_peek_last_error();
}

// forward run, loss and reverse sweep: dJ/dtheta (3*m^3) and dJ/dphi0 (ghost
// box array; interior cells hold the gradient, ghost cells are zero)
int lsmgpu_adjoint_gradient(lsmgpu_adjoint* h, double* loss, double* grad_theta,
                            double* grad_phi0) {
  const int rc = lsmgpu_adjoint_forward(h, loss);
  if (rc != LSMGPU_SUCCESS) return rc;
  return lsmgpu_adjoint_backward(h, 1.0, grad_theta, grad_phi0);
}

// reverse sweep after lsmgpu_adjoint_forward (its checkpoints and final
// state): seed * dJ/dtheta and seed * dJ/dphi0
int lsmgpu_adjoint_backward(lsmgpu_adjoint* h, double seed, double* grad_theta,
                            double* grad_phi0) {
  const char* R = "lsmgpu_adjoint_backward";
  clear_error();
  if (!h || !grad_theta || !grad_phi0) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  cudaStream_t st = cur_stream();
  cudaEvent_t e1, e2;
  cudaEventCreate(&e1);
  cudaEventCreate(&e2);
  cudaEventRecord(e1, st);
  const double vol = h->dx[0] * h->dx[1] * h->dx[2];
  k_loss<<<kLossBlocks, 256, 0, st>>>(h->phi, h->target, h->lam, h->partials, h->gb,
                                      h->fb, h->eps, vol * seed);
  ++launch_counter();
  bool ok = cuda_ok(cudaGetLastError(), R);
  const size_t m3 = (size_t)h->spl.m * h->spl.m * h->spl.m;
  for (int d = 0; ok && d < 3; d++) ok = cuda_ok(cudaMemsetAsync(h->A[d], 0, h->bytes, st), R);
  // the accumulation buffers start at zero (a failed earlier sweep may have
  // left partial sums); afterwards their consumers keep them zeroed
  ok = ok && cuda_ok(cudaMemsetAsync(h->T, 0, h->bytes, st), R) &&
       cuda_ok(cudaMemsetAsync(h->Tb, 0, h->bytes, st), R);
  ok = ok && cuda_ok(cudaMemsetAsync(h->grad_theta, 0, 3 * m3 * sizeof(double), st), R);
  const int nck = (int)h->ckpt.size();
  // the auxiliary stream starts after the forward run's checkpoints
  ok = ok && cuda_ok(cudaEventRecord(h->start, st), R) &&
       cuda_ok(cudaStreamWaitEvent(h->aux, h->start, 0), R);
  if (ok) ok = cuda_ok(recompute_segment(h, nck - 1, (nck - 1) & 1, st), R);
  for (int c = nck - 1; ok && c >= 0; c--) {
    const int b = c & 1;
    if (c > 0) {
      // segment c-1 into the other set once its last reader has finished
      const int ob = (c - 1) & 1;
      ok = cuda_ok(cudaStreamWaitEvent(h->aux, h->freed[ob], 0), R) &&
           cuda_ok(recompute_segment(h, c - 1, ob, h->aux), R) &&
           cuda_ok(cudaEventRecord(h->ready[ob], h->aux), R);
    }
    if (ok && c < nck - 1) ok = cuda_ok(cudaStreamWaitEvent(st, h->ready[b], 0), R);
    const int s0 = c * h->every, s1 = std::min(s0 + h->every, h->nsteps);
    for (int s = s1 - 1; ok && s >= s0; s--) {
      const int q = s - s0;
      const double* u = q == 0 ? h->ckpt[c] : h->segs[b][0][q];
      ok = cuda_ok(adj_step(h, u, h->segs[b][1][q], h->segs[b][2][q], st), R);
    }
    ok = ok && cuda_ok(cudaEventRecord(h->freed[b], st), R);
  }
  if (ok) {
    const int m = h->spl.m;
    k_spline_project<<<kLossBlocks, 256, 3 * m * m * m * sizeof(double), st>>>(
        h->A[0], h->A[1], h->A[2], h->grad_theta, h->spl, h->gb, h->fb, h->x_lo[0],
        h->x_lo[1], h->x_lo[2], h->dx[0], h->dx[1], h->dx[2]);
    ++launch_counter();
    ok = cuda_ok(cudaGetLastError(), R);
  }
  cudaEventRecord(e2, st);
  ok = ok && cuda_ok(cudaMemcpyAsync(grad_theta, h->grad_theta, 3 * m3 * sizeof(double),
                                     cudaMemcpyDeviceToHost, st),
                     R);
  ok = ok && cuda_ok(cudaMemcpyAsync(grad_phi0, h->lam, h->bytes, cudaMemcpyDeviceToHost, st),
                     R) &&
       cuda_ok(cudaStreamSynchronize(st), R);
  if (ok) cudaEventElapsedTime(&h->adj_ms, e1, e2);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  return ok ? LSMGPU_SUCCESS : lsmgpu_peek_last_error();
}

// device times of the last forward (including the loss) and reverse sweep
int lsmgpu_adjoint_timing(lsmgpu_adjoint* h, float* fwd_ms, float* adj_ms) {
  if (!h) return LSMGPU_ERR_NULL_POINTER;
  if (fwd_ms) *fwd_ms = h->fwd_ms;
  if (adj_ms) *adj_ms = h->adj_ms;
  return LSMGPU_SUCCESS;
}

int lsmgpu_adjoint_phi_final(lsmgpu_adjoint* h, double* host) {
  if (!h || !host) return LSMGPU_ERR_NULL_POINTER;
  return cuda_ok(cudaMemcpy(host, h->phi, h->bytes, cudaMemcpyDeviceToHost),
                 "lsmgpu_adjoint_phi_final")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}

}  // extern "C"
