// toolbox_extra.cu -- the reference's central-difference, curvature,
// external+normal, orthogonalization and subcell-fix routines as drop-in
// symbols (kernels and C ABI in one translation unit).
//
// Built with --fmad=false like toolbox_kernels.cu: each kernel evaluates the
// reference's Fortran expressions in their order with IEEE division and
// square root, so FP64 results equal the reference's bit for bit.  One
// thread per cell, x along threadIdx.x.
#include <cmath>
#include <string>

#include "capi_common.h"
#include "launch.h"

using namespace lsmgpu;

namespace {

constexpr int kBX = 32, kBY = 4;

dim3 grid_of(const FillBox& fb) {
  const unsigned gz = (unsigned)(fb.n(2) < 65535 ? fb.n(2) : 65535);
  return dim3((unsigned)((fb.n(0) + kBX - 1) / kBX), (unsigned)((fb.n(1) + kBY - 1) / kBY),
              gz);
}

#define CELLS(fb)                                                              \
  const int i = (fb).lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);     \
  const int j = (fb).lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);     \
  if (i > (fb).hi[0] || j > (fb).hi[1]) return;                                \
  for (int k = (fb).lo[2] + (int)blockIdx.z; k <= (fb).hi[2]; k += (int)gridDim.z)

template <typename T>
__device__ __forceinline__ T fmx(T a, T b) { return a > b ? a : b; }
template <typename T>
__device__ __forceinline__ T fmn(T a, T b) { return a < b ? a : b; }

// ---- lsm_spatial_derivatives3d.f.in:3016-3660 -----------------------------

// lsm3dCentralGradOrder2 (:3068-3070): (phi(+1) - phi(-1)) * (0.5/dx)
template <typename T>
__global__ void k_central_grad2(Grid3<T> gx, Grid3<T> gy, Grid3<T> gz, Grid3<const T> phi,
                                FillBox fb, T fx, T fy, T fz) {
  CELLS(fb) {
    const T* q = phi.ptr(i, j, k);
    gx(i, j, k) = (q[1] - q[-1]) * fx;
    gy(i, j, k) = (q[phi.sy] - q[-phi.sy]) * fy;
    gz(i, j, k) = (q[phi.sz] - q[-phi.sz]) * fz;
  }
}

// lsm3dCentralGradOrder4 (:3150-3158):
// (-phi(+2) + 8 phi(+1) + phi(-2) - 8 phi(-1)) * ((1/12)/dx), left to right
template <typename T>
__device__ __forceinline__ T cgrad4(const T* q, long s, T f) {
  return (-q[2 * s] + T(8) * q[s] + q[-2 * s] - T(8) * q[-s]) * f;
}
template <typename T>
__global__ void k_central_grad4(Grid3<T> gx, Grid3<T> gy, Grid3<T> gz, Grid3<const T> phi,
                                FillBox fb, T fx, T fy, T fz) {
  CELLS(fb) {
    const T* q = phi.ptr(i, j, k);
    gx(i, j, k) = cgrad4(q, 1L, fx);
    gy(i, j, k) = cgrad4(q, phi.sy, fy);
    gz(i, j, k) = cgrad4(q, phi.sz, fz);
  }
}

// lsm3dLaplacianOrder2 (:3244-3250), 1/dx/dx per axis
template <typename T>
__global__ void k_laplacian2(Grid3<T> lap, Grid3<const T> phi, FillBox fb, T ix, T iy,
                             T iz) {
  CELLS(fb) {
    const T* q = phi.ptr(i, j, k);
    lap(i, j, k) = ix * (q[1] - T(2) * q[0] + q[-1]) +
                   iy * (q[phi.sy] - T(2) * q[0] + q[-phi.sy]) +
                   iz * (q[phi.sz] - T(2) * q[0] + q[-phi.sz]);
  }
}

// lsm3dPhiUpwindGradF (:3324-3470): per axis, the one-sided derivative of F
// toward the neighbour nearer the interface; cells with phi == 0 untouched
template <typename T>
__device__ __forceinline__ void upwind_gradf(T* out, T pc, T pm, T pp, T fp, T fm) {
  if (pc > T(0)) {
    if (pm <= pc) *out = (pp < pm) ? fp : fm;
    else if (pp <= pc) *out = fp;
    else *out = T(0);
  } else if (pc < T(0)) {
    if (pm >= pc) *out = (pp > pm) ? fp : fm;
    else if (pp >= pc) *out = fp;
    else *out = T(0);
  }
}
template <typename T>
__global__ void k_phi_upwind_grad_f(Grid3<T> Fx, Grid3<T> Fy, Grid3<T> Fz,
                                    Grid3<const T> Fxp, Grid3<const T> Fyp,
                                    Grid3<const T> Fzp, Grid3<const T> Fxm,
                                    Grid3<const T> Fym, Grid3<const T> Fzm,
                                    Grid3<const T> phi, FillBox fb) {
  CELLS(fb) {
    const T* q = phi.ptr(i, j, k);
    const T pc = q[0];
    upwind_gradf(Fx.ptr(i, j, k), pc, q[-1], q[1], Fxp(i, j, k), Fxm(i, j, k));
    upwind_gradf(Fy.ptr(i, j, k), pc, q[-phi.sy], q[phi.sy], Fyp(i, j, k), Fym(i, j, k));
    upwind_gradf(Fz.ptr(i, j, k), pc, q[-phi.sz], q[phi.sz], Fzp(i, j, k), Fzm(i, j, k));
  }
}

// lsm3dAverageGradPhi (:3561-3566)
template <typename T>
__global__ void k_average_grad(Grid3<T> gx, Grid3<T> gy, Grid3<T> gz, Grid3<const T> xp,
                               Grid3<const T> yp, Grid3<const T> zp, Grid3<const T> xm,
                               Grid3<const T> ym, Grid3<const T> zm, FillBox fb) {
  CELLS(fb) {
    gx(i, j, k) = T(0.5) * (xp(i, j, k) + xm(i, j, k));
    gy(i, j, k) = T(0.5) * (yp(i, j, k) + ym(i, j, k));
    gz(i, j, k) = T(0.5) * (zp(i, j, k) + zm(i, j, k));
  }
}

// lsm3dGradientMagnitude (:3626-3651): squares and magnitude below 1e-8 are 0
template <typename T>
__global__ void k_gradient_magnitude(Grid3<const T> gx, Grid3<const T> gy,
                                     Grid3<const T> gz, Grid3<T> mag, FillBox fb) {
  CELLS(fb) {
    const T tol = T(1.0e-8);
    const T x = gx(i, j, k), y = gy(i, j, k), z = gz(i, j, k);
    T sx = x * x, sy = y * y, sz = z * z;
    if (sx < tol) sx = T(0);
    if (sy < tol) sy = T(0);
    if (sz < tol) sz = T(0);
    const T t = sqrtT(sx + sy + sz);
    mag(i, j, k) = (t < tol) ? T(0) : t;
  }
}

// ---- lsm_level_set_evolution3d.f.in:356-710 -------------------------------

// lsm3dAddConstCurvTermToLSERHS (:431-452)
template <typename T>
__global__ void k_add_const_curv(Grid3<T> rhs, Grid3<const T> px, Grid3<const T> py,
                                 Grid3<const T> pz, Grid3<const T> pxx, Grid3<const T> pxy,
                                 Grid3<const T> pxz, Grid3<const T> pyy, Grid3<const T> pyz,
                                 Grid3<const T> pzz, FillBox fb, T b) {
  CELLS(fb) {
    const T x = px(i, j, k), y = py(i, j, k), z = pz(i, j, k);
    const T g2 = x * x + y * y + z * z;
    T curv;
    if (g2 < Consts<T>::zero_tol) {
      curv = T(0);
    } else {
      const T xx = pxx(i, j, k), yy = pyy(i, j, k), zz = pzz(i, j, k);
      curv = xx * y * y + yy * x * x - T(2) * pxy(i, j, k) * x * y + xx * z * z +
             zz * x * x - T(2) * pxz(i, j, k) * x * z + yy * z * z + zz * y * y -
             T(2) * pyz(i, j, k) * y * z;
      curv = curv / g2;
    }
    rhs(i, j, k) = rhs(i, j, k) + b * curv;
  }
}

// The two terms below run the reference's loop nest k over [klo_fb, khi_gb],
// j over [jlo_fb, jhi_gb], i over [ilo_gb, ihi_gb] of the RHS array
// (:505-507, :586-588); ``box`` is that region.

// lsm3dAddConstPrecomputedCurvTermToLSERHS (:509-510)
template <typename T>
__global__ void k_add_precomputed_curv(Grid3<T> rhs, Grid3<const T> kappa,
                                       Grid3<const T> mag, FillBox box, T b) {
  CELLS(box) { rhs(i, j, k) = rhs(i, j, k) + b * kappa(i, j, k) * mag(i, j, k); }
}

// lsm3dAddExternalAndNormalVelTermToLSERHS (:593-684): Godunov choice per
// axis for H = V.grad phi + Vn |grad phi|, then the RHS update
template <typename T>
__device__ __forceinline__ T ext_normal_pick(T v, T vn, T dp, T dm) {
  const T hp = v + vn * dp, hm = v + vn * dm;
  if (hp > T(0)) {
    if (hm > T(0)) return dm;
    return -(v / vn);
  }
  if (hm < T(0)) return dp;
  return (fabsT(hp) > fabsT(hm)) ? dp : dm;
}
template <typename T>
__global__ void k_add_ext_normal(Grid3<T> rhs, Grid3<const T> xp, Grid3<const T> yp,
                                 Grid3<const T> zp, Grid3<const T> xm, Grid3<const T> ym,
                                 Grid3<const T> zm, Grid3<const T> vn, Grid3<const T> vx,
                                 Grid3<const T> vy, Grid3<const T> vz, FillBox box) {
  CELLS(box) {
    const T n = vn(i, j, k), x = vx(i, j, k), y = vy(i, j, k), z = vz(i, j, k);
    const T gx = ext_normal_pick(x, n, xp(i, j, k), xm(i, j, k));
    const T gy = ext_normal_pick(y, n, yp(i, j, k), ym(i, j, k));
    const T gz = ext_normal_pick(z, n, zp(i, j, k), zm(i, j, k));
    const T nsq = gx * gx + gy * gy + gz * gz;
    if (fabsT(n) >= Consts<T>::zero_tol && nsq >= Consts<T>::zero_tol)
      rhs(i, j, k) = rhs(i, j, k) - x * gx - y * gy - z * gz - n * sqrtT(nsq);
    else
      rhs(i, j, k) = rhs(i, j, k) - x * gx - y * gy - z * gz;
  }
}

// ---- lsm_reinitialization3d.f.in:296-754 ----------------------------------

// lsm3dComputeOrthogonalizationEqnRHS (:416-457)
template <typename T>
__global__ void k_ortho_rhs(Grid3<T> rhs, Grid3<const T> pxp, Grid3<const T> pyp,
                            Grid3<const T> pzp, Grid3<const T> pxm, Grid3<const T> pym,
                            Grid3<const T> pzm, Grid3<const T> psi, Grid3<const T> sxp,
                            Grid3<const T> syp, Grid3<const T> szp, Grid3<const T> sxm,
                            Grid3<const T> sym, Grid3<const T> szm, FillBox fb, T dx_sq) {
  CELLS(fb) {
    const T g1 = T(0.5) * (sxp(i, j, k) + sxm(i, j, k));
    const T g2 = T(0.5) * (syp(i, j, k) + sym(i, j, k));
    const T g3 = T(0.5) * (szp(i, j, k) + szm(i, j, k));
    T nrm = g1 * g1 + g2 * g2 + g3 * g3;
    nrm = sqrtT(nrm);
    const T ps = psi(i, j, k);
    if (fabsT(ps) > Consts<T>::zero_tol && nrm > Consts<T>::zero_tol) {
      const T sgn = ps / sqrtT(ps * ps + dx_sq * (nrm * nrm));
      rhs(i, j, k) = -(T(1) / nrm *
                       (fmx(sgn * g1, T(0)) * pxm(i, j, k) + fmn(sgn * g1, T(0)) * pxp(i, j, k) +
                        fmx(sgn * g2, T(0)) * pym(i, j, k) + fmn(sgn * g2, T(0)) * pyp(i, j, k) +
                        fmx(sgn * g3, T(0)) * pzm(i, j, k) + fmn(sgn * g3, T(0)) * pzp(i, j, k)));
    } else {
      rhs(i, j, k) = T(0);
    }
  }
}

// lsm3dComputeDistanceForSubcellFix (:521-571)
template <typename T>
__device__ __forceinline__ bool sign_change(T a, T c) {
  return (a > T(0) && c <= T(0)) || (a <= T(0) && c > T(0));
}
template <typename T>
__global__ void k_distance_subcell(Grid3<T> dist, Grid3<const T> phi0, FillBox fb, T flag) {
  CELLS(fb) {
    const T* q = phi0.ptr(i, j, k);
    const T c = q[0];
    const long s[3] = {1L, phi0.sy, phi0.sz};
    bool near = false;
#pragma unroll
    for (int d = 0; d < 3; d++) near = near || sign_change(q[s[d]], c) || sign_change(q[-s[d]], c);
    if (!near) {
      dist(i, j, k) = flag;
    } else {
      T delta = Consts<T>::zero_tol;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const T d1 = fabsT(q[s[d]] - q[-s[d]]) / T(2);
        const T d2 = fabsT(q[s[d]] - c);
        const T d3 = fabsT(c - q[-s[d]]);
        delta = fmx(fmx(fmx(d1, d2), d3), delta);
      }
      dist(i, j, k) = c / delta;
    }
  }
}

// lsm3dComputeReinitializationEqnRHSSubcellFixOrder1 (:660-726)
template <typename T>
__global__ void k_reinit_subcell(Grid3<T> rhs, Grid3<const T> phi, Grid3<const T> phi0,
                                 Grid3<const T> dist, Grid3<const T> pxp, Grid3<const T> pyp,
                                 Grid3<const T> pzp, Grid3<const T> pxm, Grid3<const T> pym,
                                 Grid3<const T> pzm, FillBox fb, T flag, T max_dx) {
  CELLS(fb) {
    const T p0 = phi0(i, j, k);
    const T sgn0 = fabsT(p0) > Consts<T>::zero_tol ? copysign(T(1), p0) : T(0);
    const T pc = phi(i, j, k);
    const T d0 = dist(i, j, k);
    if (d0 == flag) {
      T gp[3] = {pxp(i, j, k), pyp(i, j, k), pzp(i, j, k)};
      T gm[3] = {pxm(i, j, k), pym(i, j, k), pzm(i, j, k)};
      T gs[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (pc > T(0)) {
          gp[d] = fmx(-gp[d], T(0));
          gm[d] = fmx(gm[d], T(0));
        } else {
          gp[d] = fmx(gp[d], T(0));
          gm[d] = fmx(-gm[d], T(0));
        }
        gs[d] = fmx(gp[d], gm[d]);
      }
      if (fabsT(pc) > Consts<T>::zero_tol) {
        const T nsq = gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2];
        rhs(i, j, k) = sgn0 - sgn0 * sqrtT(nsq);
      } else {
        rhs(i, j, k) = T(0);
      }
    } else {
      rhs(i, j, k) = d0 - sgn0 * fabsT(pc) / max_dx;
    }
  }
}

#undef CELLS

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using R_ = LSMLIB_REAL;
const int kReal = (int)sizeof(R_);

bool fb_empty(const FillBox& fb) {
  return fb.hi[0] < fb.lo[0] || fb.hi[1] < fb.lo[1] || fb.hi[2] < fb.lo[2];
}

// fill box grown by w cells (per axis) lies inside box b: the cells a
// routine reads
bool reads_inside(const Box& b, const FillBox& fb, int w, const char* what,
                  const char* R) {
  return box_valid(b, what, R) && covers(b, fb, w, what, R);
}

// one call: validation done by the caller, arrays added here
struct Call {
  const char* R;
  Staging s;
  bool ok = true;
  explicit Call(const char* r) : R(r), s(cur_stream()) {}
  template <typename P>
  Grid3<R_> out(P* p, const Box& b, const char* what, Role role = kOut) {
    void* d = ok ? s.add(p, b, kReal, role, what, R) : nullptr;
    ok = ok && d;
    return make_grid((R_*)d, b);
  }
  Grid3<const R_> in(const R_* p, const Box& b, const char* what) {
    void* d = ok ? s.add(p, b, kReal, kIn, what, R) : nullptr;
    ok = ok && d;
    return make_grid((const R_*)d, b);
  }
  void finish() {
    if (ok && cuda_ok(cudaGetLastError(), R)) s.finish(R);
  }
};

#define BOX(p) box_from(ilo_##p, ihi_##p, jlo_##p, jhi_##p, klo_##p, khi_##p)
#define FB() fill_from(ilo_fb, ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb)
#define NULLCHK(...)                                                        \
  do {                                                                      \
    const void* ps_[] = {__VA_ARGS__};                                      \
    for (const void* p_ : ps_)                                              \
      if (!p_) {                                                            \
        set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument pointer"); \
        return;                                                             \
      }                                                                     \
  } while (0)
#define B6(p) ilo_##p, ihi_##p, jlo_##p, jhi_##p, klo_##p, khi_##p
#define LAUNCH(kernel, fb, ...)                                             \
  do {                                                                      \
    kernel<R_><<<grid_of(fb), dim3(kBX, kBY), 0, cur_stream()>>>(__VA_ARGS__); \
    ++launch_counter();                                                     \
  } while (0)

R_ max3(R_ a, R_ b, R_ c) {
  R_ m = a > b ? a : b;
  return m > c ? m : c;
}

// region of the reference's loop nest in the precomputed-curvature and
// external+normal terms: i over the RHS ghost box, j and k from the fill box's
// lower bound to the RHS ghost box's upper bound
FillBox odd_region(const Box& grhs, const FillBox& fb) {
  FillBox r;
  r.lo[0] = grhs.lo[0]; r.hi[0] = grhs.hi(0);
  r.lo[1] = fb.lo[1];   r.hi[1] = grhs.hi(1);
  r.lo[2] = fb.lo[2];   r.hi[2] = grhs.hi(2);
  return r;
}

}  // namespace

extern "C" {

void lsm3dcentralgradorder2_(R_* phi_x, R_* phi_y, R_* phi_z, LSMGPU_BOX6(g), const R_* phi,
                             LSMGPU_BOX6(phi), LSMGPU_BOX6(fb), const R_* dx, const R_* dy,
                             const R_* dz) {
  const char* R = "LSM3D_CENTRAL_GRAD_ORDER2";
  clear_error();
  NULLCHK(B6(g), B6(phi), B6(fb), dx, dy, dz);
  const Box g = BOX(g), gp = BOX(phi);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(g, fb, 0, "grad_phi", R) || !reads_inside(gp, fb, 1, "phi", R)) return;
  Call c(R);
  auto x = c.out(phi_x, g, "phi_x"), y = c.out(phi_y, g, "phi_y"), z = c.out(phi_z, g, "phi_z");
  auto p = c.in(phi, gp, "phi");
  if (!c.ok) return;
  LAUNCH(k_central_grad2, fb, x, y, z, p, fb, 0.5 / *dx, 0.5 / *dy, 0.5 / *dz);
  c.finish();
}

void lsm3dcentralgradorder4_(R_* phi_x, R_* phi_y, R_* phi_z, LSMGPU_BOX6(g), const R_* phi,
                             LSMGPU_BOX6(phi), LSMGPU_BOX6(fb), const R_* dx, const R_* dy,
                             const R_* dz) {
  const char* R = "LSM3D_CENTRAL_GRAD_ORDER4";
  clear_error();
  NULLCHK(B6(g), B6(phi), B6(fb), dx, dy, dz);
  const Box g = BOX(g), gp = BOX(phi);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(g, fb, 0, "grad_phi", R) || !reads_inside(gp, fb, 2, "phi", R)) return;
  Call c(R);
  auto x = c.out(phi_x, g, "phi_x"), y = c.out(phi_y, g, "phi_y"), z = c.out(phi_z, g, "phi_z");
  auto p = c.in(phi, gp, "phi");
  if (!c.ok) return;
  const R_ f = 0.0833333333333333333333;
  LAUNCH(k_central_grad4, fb, x, y, z, p, fb, f / *dx, f / *dy, f / *dz);
  c.finish();
}

void lsm3dlaplacianorder2_(R_* laplacian_phi, LSMGPU_BOX6(l), const R_* phi,
                           LSMGPU_BOX6(phi), LSMGPU_BOX6(fb), const R_* dx, const R_* dy,
                           const R_* dz) {
  const char* R = "LSM3D_LAPLACIAN_ORDER2";
  clear_error();
  NULLCHK(B6(l), B6(phi), B6(fb), dx, dy, dz);
  const Box gl = BOX(l), gp = BOX(phi);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(gl, fb, 0, "laplacian_phi", R) || !reads_inside(gp, fb, 1, "phi", R))
    return;
  Call c(R);
  auto l = c.out(laplacian_phi, gl, "laplacian_phi");
  auto p = c.in(phi, gp, "phi");
  if (!c.ok) return;
  LAUNCH(k_laplacian2, fb, l, p, fb, 1.0 / *dx / *dx, 1.0 / *dy / *dy, 1.0 / *dz / *dz);
  c.finish();
}

void lsm3dphiupwindgradf_(R_* F_x, R_* F_y, R_* F_z, LSMGPU_BOX6(g), const R_* F_x_plus,
                          const R_* F_y_plus, const R_* F_z_plus, LSMGPU_BOX6(gp),
                          const R_* F_x_minus, const R_* F_y_minus, const R_* F_z_minus,
                          LSMGPU_BOX6(gm), const R_* phi, LSMGPU_BOX6(phi),
                          LSMGPU_BOX6(fb)) {
  const char* R = "LSM3D_PHI_UPWIND_GRAD_F";
  clear_error();
  NULLCHK(B6(g), B6(gp), B6(gm), B6(phi), B6(fb));
  const Box g = BOX(g), gpl = BOX(gp), gmi = BOX(gm), gph = BOX(phi);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(g, fb, 0, "grad_F", R) || !reads_inside(gpl, fb, 0, "grad_F_plus", R) ||
      !reads_inside(gmi, fb, 0, "grad_F_minus", R) || !reads_inside(gph, fb, 1, "phi", R))
    return;
  Call c(R);
  // outputs keep their values where phi == 0
  auto x = c.out(F_x, g, "F_x", kInOut), y = c.out(F_y, g, "F_y", kInOut),
       z = c.out(F_z, g, "F_z", kInOut);
  auto xp = c.in(F_x_plus, gpl, "F_x_plus"), yp = c.in(F_y_plus, gpl, "F_y_plus"),
       zp = c.in(F_z_plus, gpl, "F_z_plus");
  auto xm = c.in(F_x_minus, gmi, "F_x_minus"), ym = c.in(F_y_minus, gmi, "F_y_minus"),
       zm = c.in(F_z_minus, gmi, "F_z_minus");
  auto p = c.in(phi, gph, "phi");
  if (!c.ok) return;
  LAUNCH(k_phi_upwind_grad_f, fb, x, y, z, xp, yp, zp, xm, ym, zm, p, fb);
  c.finish();
}

void lsm3daveragegradphi_(R_* phi_x, R_* phi_y, R_* phi_z, LSMGPU_BOX6(g),
                          const R_* phi_x_plus, const R_* phi_y_plus, const R_* phi_z_plus,
                          LSMGPU_BOX6(gp), const R_* phi_x_minus, const R_* phi_y_minus,
                          const R_* phi_z_minus, LSMGPU_BOX6(gm), LSMGPU_BOX6(fb)) {
  const char* R = "LSM3D_AVERAGE_GRAD_PHI";
  clear_error();
  NULLCHK(B6(g), B6(gp), B6(gm), B6(fb));
  const Box g = BOX(g), gpl = BOX(gp), gmi = BOX(gm);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(g, fb, 0, "grad_phi", R) || !reads_inside(gpl, fb, 0, "grad_phi_plus", R) ||
      !reads_inside(gmi, fb, 0, "grad_phi_minus", R))
    return;
  Call c(R);
  auto x = c.out(phi_x, g, "phi_x"), y = c.out(phi_y, g, "phi_y"), z = c.out(phi_z, g, "phi_z");
  auto xp = c.in(phi_x_plus, gpl, "phi_x_plus"), yp = c.in(phi_y_plus, gpl, "phi_y_plus"),
       zp = c.in(phi_z_plus, gpl, "phi_z_plus");
  auto xm = c.in(phi_x_minus, gmi, "phi_x_minus"), ym = c.in(phi_y_minus, gmi, "phi_y_minus"),
       zm = c.in(phi_z_minus, gmi, "phi_z_minus");
  if (!c.ok) return;
  LAUNCH(k_average_grad, fb, x, y, z, xp, yp, zp, xm, ym, zm, fb);
  c.finish();
}

void lsm3dgradientmagnitude_(const R_* phi_x, const R_* phi_y, const R_* phi_z,
                             R_* grad_phi_mag, LSMGPU_BOX6(g), LSMGPU_BOX6(fb)) {
  const char* R = "LSM3D_GRADIENT_MAGNITUDE";
  clear_error();
  NULLCHK(B6(g), B6(fb));
  const Box g = BOX(g);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(g, fb, 0, "grad_phi", R)) return;
  Call c(R);
  auto x = c.in(phi_x, g, "phi_x"), y = c.in(phi_y, g, "phi_y"), z = c.in(phi_z, g, "phi_z");
  auto m = c.out(grad_phi_mag, g, "grad_phi_mag");
  if (!c.ok) return;
  LAUNCH(k_gradient_magnitude, fb, x, y, z, m, fb);
  c.finish();
}

void lsm3daddconstcurvtermtolserhs_(R_* lse_rhs, LSMGPU_BOX6(r), const R_* phi_x,
                                    const R_* phi_y, const R_* phi_z, LSMGPU_BOX6(g1),
                                    const R_* phi_xx, const R_* phi_xy, const R_* phi_xz,
                                    const R_* phi_yy, const R_* phi_yz, const R_* phi_zz,
                                    LSMGPU_BOX6(g2), const R_* b, LSMGPU_BOX6(fb)) {
  const char* R = "LSM3D_ADD_CONST_CURV_TERM_TO_LSE_RHS";
  clear_error();
  NULLCHK(B6(r), B6(g1), B6(g2), b, B6(fb));
  const Box gr = BOX(r), ga = BOX(g1), gb = BOX(g2);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(gr, fb, 0, "lse_rhs", R) || !reads_inside(ga, fb, 0, "grad_phi", R) ||
      !reads_inside(gb, fb, 0, "grad2_phi", R))
    return;
  Call c(R);
  auto rr = c.out(lse_rhs, gr, "lse_rhs", kInOut);
  auto x = c.in(phi_x, ga, "phi_x"), y = c.in(phi_y, ga, "phi_y"), z = c.in(phi_z, ga, "phi_z");
  auto xx = c.in(phi_xx, gb, "phi_xx"), xy = c.in(phi_xy, gb, "phi_xy"),
       xz = c.in(phi_xz, gb, "phi_xz"), yy = c.in(phi_yy, gb, "phi_yy"),
       yz = c.in(phi_yz, gb, "phi_yz"), zz = c.in(phi_zz, gb, "phi_zz");
  if (!c.ok) return;
  LAUNCH(k_add_const_curv, fb, rr, x, y, z, xx, xy, xz, yy, yz, zz, fb, *b);
  c.finish();
}

void lsm3daddconstprecomputedcurvtermtolserhs_(R_* lse_rhs, LSMGPU_BOX6(r), const R_* kappa,
                                               LSMGPU_BOX6(kap), const R_* grad_phi_mag,
                                               LSMGPU_BOX6(g), const R_* b, LSMGPU_BOX6(fb)) {
  const char* R = "LSM3D_ADD_CONST_PRECOMPUTED_CURV_TERM_TO_LSE_RHS";
  clear_error();
  NULLCHK(B6(r), B6(kap), B6(g), b, B6(fb));
  const Box gr = BOX(r), gk = BOX(kap), gg = BOX(g);
  if (!box_valid(gr, "lse_rhs", R)) return;
  const FillBox box = odd_region(gr, FB());
  if (fb_empty(box)) return;
  if (!reads_inside(gk, box, 0, "kappa", R) || !reads_inside(gg, box, 0, "grad_phi_mag", R))
    return;
  Call c(R);
  auto rr = c.out(lse_rhs, gr, "lse_rhs", kInOut);
  auto kk = c.in(kappa, gk, "kappa"), mm = c.in(grad_phi_mag, gg, "grad_phi_mag");
  if (!c.ok) return;
  LAUNCH(k_add_precomputed_curv, box, rr, kk, mm, box, *b);
  c.finish();
}

void lsm3daddexternalandnormalveltermtolserhs_(
    R_* lse_rhs, LSMGPU_BOX6(r), const R_* phi_x_plus, const R_* phi_y_plus,
    const R_* phi_z_plus, LSMGPU_BOX6(gp), const R_* phi_x_minus, const R_* phi_y_minus,
    const R_* phi_z_minus, LSMGPU_BOX6(gm), const R_* vel_n, const R_* vel_x,
    const R_* vel_y, const R_* vel_z, LSMGPU_BOX6(v), LSMGPU_BOX6(fb)) {
  const char* R = "LSM3D_ADD_EXTERNAL_AND_NORMAL_VEL_TERM_TO_LSE_RHS";
  clear_error();
  NULLCHK(B6(r), B6(gp), B6(gm), B6(v), B6(fb));
  const Box gr = BOX(r), gpl = BOX(gp), gmi = BOX(gm), gv = BOX(v);
  if (!box_valid(gr, "lse_rhs", R)) return;
  const FillBox box = odd_region(gr, FB());
  if (fb_empty(box)) return;
  if (!reads_inside(gpl, box, 0, "grad_phi_plus", R) ||
      !reads_inside(gmi, box, 0, "grad_phi_minus", R) || !reads_inside(gv, box, 0, "vel", R))
    return;
  Call c(R);
  auto rr = c.out(lse_rhs, gr, "lse_rhs", kInOut);
  auto xp = c.in(phi_x_plus, gpl, "phi_x_plus"), yp = c.in(phi_y_plus, gpl, "phi_y_plus"),
       zp = c.in(phi_z_plus, gpl, "phi_z_plus");
  auto xm = c.in(phi_x_minus, gmi, "phi_x_minus"), ym = c.in(phi_y_minus, gmi, "phi_y_minus"),
       zm = c.in(phi_z_minus, gmi, "phi_z_minus");
  auto n = c.in(vel_n, gv, "vel_n"), x = c.in(vel_x, gv, "vel_x"), y = c.in(vel_y, gv, "vel_y"),
       z = c.in(vel_z, gv, "vel_z");
  if (!c.ok) return;
  LAUNCH(k_add_ext_normal, box, rr, xp, yp, zp, xm, ym, zm, n, x, y, z, box);
  c.finish();
}

void lsm3dcomputeorthogonalizationeqnrhs_(
    R_* ortho_rhs, LSMGPU_BOX6(r), const R_* phi_x_plus, const R_* phi_y_plus,
    const R_* phi_z_plus, LSMGPU_BOX6(gp), const R_* phi_x_minus, const R_* phi_y_minus,
    const R_* phi_z_minus, LSMGPU_BOX6(gm), const R_* psi, LSMGPU_BOX6(psi),
    const R_* psi_x_plus, const R_* psi_y_plus, const R_* psi_z_plus, LSMGPU_BOX6(sp),
    const R_* psi_x_minus, const R_* psi_y_minus, const R_* psi_z_minus, LSMGPU_BOX6(sm),
    LSMGPU_BOX6(fb), const R_* dx, const R_* dy, const R_* dz) {
  const char* R = "LSM3D_COMPUTE_ORTHOGONALIZATION_EQN_RHS";
  clear_error();
  NULLCHK(B6(r), B6(gp), B6(gm), B6(psi), B6(sp), B6(sm), B6(fb), dx, dy, dz);
  const Box gr = BOX(r), gpl = BOX(gp), gmi = BOX(gm), gps = BOX(psi), gsp = BOX(sp),
            gsm = BOX(sm);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(gr, fb, 0, "ortho_rhs", R) || !reads_inside(gpl, fb, 0, "grad_phi_plus", R) ||
      !reads_inside(gmi, fb, 0, "grad_phi_minus", R) || !reads_inside(gps, fb, 0, "psi", R) ||
      !reads_inside(gsp, fb, 0, "grad_psi_plus", R) ||
      !reads_inside(gsm, fb, 0, "grad_psi_minus", R))
    return;
  Call c(R);
  auto rr = c.out(ortho_rhs, gr, "ortho_rhs");
  auto xp = c.in(phi_x_plus, gpl, "phi_x_plus"), yp = c.in(phi_y_plus, gpl, "phi_y_plus"),
       zp = c.in(phi_z_plus, gpl, "phi_z_plus");
  auto xm = c.in(phi_x_minus, gmi, "phi_x_minus"), ym = c.in(phi_y_minus, gmi, "phi_y_minus"),
       zm = c.in(phi_z_minus, gmi, "phi_z_minus");
  auto ps = c.in(psi, gps, "psi");
  auto sxp = c.in(psi_x_plus, gsp, "psi_x_plus"), syp = c.in(psi_y_plus, gsp, "psi_y_plus"),
       szp = c.in(psi_z_plus, gsp, "psi_z_plus");
  auto sxm = c.in(psi_x_minus, gsm, "psi_x_minus"), sym = c.in(psi_y_minus, gsm, "psi_y_minus"),
       szm = c.in(psi_z_minus, gsm, "psi_z_minus");
  if (!c.ok) return;
  R_ dx_sq = max3(*dx, *dy, *dz);
  dx_sq = dx_sq * dx_sq;
  LAUNCH(k_ortho_rhs, fb, rr, xp, yp, zp, xm, ym, zm, ps, sxp, syp, szp, sxm, sym, szm, fb,
         dx_sq);
  c.finish();
}

void lsm3dcomputedistanceforsubcellfix_(R_* distance0, const R_* phi0, LSMGPU_BOX6(p),
                                        LSMGPU_BOX6(fb), const R_* dx, const R_* dy,
                                        const R_* dz) {
  const char* R = "LSM3D_COMPUTE_DISTANCE_FOR_SUBCELL_FIX";
  clear_error();
  NULLCHK(B6(p), B6(fb), dx, dy, dz);
  const Box gp = BOX(p);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(gp, fb, 1, "phi0", R)) return;
  Call c(R);
  auto d = c.out(distance0, gp, "distance0");
  auto p0 = c.in(phi0, gp, "phi0");
  if (!c.ok) return;
  LAUNCH(k_distance_subcell, fb, d, p0, fb, -1000.0 * max3(*dx, *dy, *dz));
  c.finish();
}

void lsm3dcomputereinitializationeqnrhssubcellfixorder1_(
    R_* reinit_rhs, LSMGPU_BOX6(r), const R_* phi, LSMGPU_BOX6(phi), const R_* phi0,
    const R_* distance0, LSMGPU_BOX6(p0), const R_* phi_x_plus, const R_* phi_y_plus,
    const R_* phi_z_plus, LSMGPU_BOX6(gp), const R_* phi_x_minus, const R_* phi_y_minus,
    const R_* phi_z_minus, LSMGPU_BOX6(gm), LSMGPU_BOX6(fb), const R_* dx, const R_* dy,
    const R_* dz) {
  const char* R = "LSM3D_COMPUTE_REINITIALIZATION_EQN_RHS_SUBCELL_FIX_ORDER1";
  clear_error();
  NULLCHK(B6(r), B6(phi), B6(p0), B6(gp), B6(gm), B6(fb), dx, dy, dz);
  const Box gr = BOX(r), gph = BOX(phi), g0 = BOX(p0), gpl = BOX(gp), gmi = BOX(gm);
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  if (!reads_inside(gr, fb, 0, "reinit_rhs", R) || !reads_inside(gph, fb, 0, "phi", R) ||
      !reads_inside(g0, fb, 0, "phi0", R) || !reads_inside(gpl, fb, 0, "grad_phi_plus", R) ||
      !reads_inside(gmi, fb, 0, "grad_phi_minus", R))
    return;
  Call c(R);
  auto rr = c.out(reinit_rhs, gr, "reinit_rhs");
  auto p = c.in(phi, gph, "phi"), p0 = c.in(phi0, g0, "phi0"), d0 = c.in(distance0, g0, "distance0");
  auto xp = c.in(phi_x_plus, gpl, "phi_x_plus"), yp = c.in(phi_y_plus, gpl, "phi_y_plus"),
       zp = c.in(phi_z_plus, gpl, "phi_z_plus");
  auto xm = c.in(phi_x_minus, gmi, "phi_x_minus"), ym = c.in(phi_y_minus, gmi, "phi_y_minus"),
       zm = c.in(phi_z_minus, gmi, "phi_z_minus");
  if (!c.ok) return;
  const R_ max_dx = max3(*dx, *dy, *dz);
  LAUNCH(k_reinit_subcell, fb, rr, p, p0, d0, xp, yp, zp, xm, ym, zm, fb, -1000.0 * max_dx,
         max_dx);
  c.finish();
}

}  // extern "C"
