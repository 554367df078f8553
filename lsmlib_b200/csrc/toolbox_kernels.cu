// toolbox_kernels.cu -- one CUDA kernel per reference toolbox routine.
//
// This translation unit is compiled with --fmad=false: every kernel evaluates
// the reference's Fortran expressions in the reference's order with IEEE
// division and square root, so the FP64 results equal the reference's FP64
// build bit for bit.  One thread computes one fill-box cell; the x index runs
// along threadIdx.x so that every array access of a warp is coalesced.
#include <cstdio>

#include "launch.h"
#include "stencil.cuh"

namespace lsmgpu {

unsigned long long& launch_counter() {
  static unsigned long long n = 0;
  return n;
}

namespace {

constexpr int kBX = 32, kBY = 4;

inline dim3 cell_grid(const FillBox& fb) {
  unsigned gz = (unsigned)(fb.n(2) < 65535 ? fb.n(2) : 65535);
  return dim3((unsigned)((fb.n(0) + kBX - 1) / kBX),
              (unsigned)((fb.n(1) + kBY - 1) / kBY), gz);
}

inline cudaError_t post_launch() {
  ++launch_counter();
  return cudaGetLastError();
}

#define CELL_LOOP_BEGIN(fb)                                              \
  const int i = (fb).lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x); \
  const int j = (fb).lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y); \
  if (i > (fb).hi[0] || j > (fb).hi[1]) return;                          \
  for (int k = (fb).lo[2] + (int)blockIdx.z; k <= (fb).hi[2];            \
       k += (int)gridDim.z) {
#define CELL_LOOP_END }

// ---------------------------------------------------------------------------
// plus/minus gradients: LSM3D_HJ_ENO1/2/3, LSM3D_HJ_WENO5
// ---------------------------------------------------------------------------
template <int SCHEME, typename T>
__global__ void __launch_bounds__(128)
k_hj_plus_minus(Grid3<T> xp, Grid3<T> yp, Grid3<T> zp, Grid3<T> xm,
                Grid3<T> ym, Grid3<T> zm, Grid3<const T> phi, FillBox fb,
                T ix, T iy, T iz) {
  CELL_LOOP_BEGIN(fb)
  const T* q = phi.ptr(i, j, k);
  xp(i, j, k) = plus_strict<SCHEME>(q, 1L, ix);
  xm(i, j, k) = minus_strict<SCHEME>(q, 1L, ix);
  yp(i, j, k) = plus_strict<SCHEME>(q, phi.sy, iy);
  ym(i, j, k) = minus_strict<SCHEME>(q, phi.sy, iy);
  zp(i, j, k) = plus_strict<SCHEME>(q, phi.sz, iz);
  zm(i, j, k) = minus_strict<SCHEME>(q, phi.sz, iz);
  CELL_LOOP_END
}

// ---------------------------------------------------------------------------
// upwind gradients: LSM3D_UPWIND_HJ_ENO1/2/3, LSM3D_UPWIND_HJ_WENO5
// |v| < zero_tol -> 0; v > 0 -> minus value; else plus value
// (lsm_spatial_derivatives3d.f.in:2756-2776)
// ---------------------------------------------------------------------------
template <int SCHEME, typename T>
__device__ __forceinline__ T upwind_one(const T* q, long s, T inv, T v) {
  if (fabsT(v) < Consts<T>::zero_tol) return T(0);
  if (v > T(0)) return minus_strict<SCHEME>(q, s, inv);
  return plus_strict<SCHEME>(q, s, inv);
}

template <int SCHEME, typename T>
__global__ void __launch_bounds__(128)
k_hj_upwind(Grid3<T> gx, Grid3<T> gy, Grid3<T> gz, Grid3<const T> phi,
            Grid3<const T> vx, Grid3<const T> vy, Grid3<const T> vz,
            FillBox fb, T ix, T iy, T iz) {
  CELL_LOOP_BEGIN(fb)
  const T* q = phi.ptr(i, j, k);
  gx(i, j, k) = upwind_one<SCHEME>(q, 1L, ix, ld(vx.ptr(i, j, k)));
  gy(i, j, k) = upwind_one<SCHEME>(q, phi.sy, iy, ld(vy.ptr(i, j, k)));
  gz(i, j, k) = upwind_one<SCHEME>(q, phi.sz, iz, ld(vz.ptr(i, j, k)));
  CELL_LOOP_END
}

// ---------------------------------------------------------------------------
// pointwise kernels
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_fill(T* p, long n, T v) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x)
    p[t] = v;
}

// lsm_level_set_evolution3d.f.in:84-87
template <typename T>
__global__ void __launch_bounds__(128)
k_add_advection(Grid3<T> rhs, Grid3<const T> px, Grid3<const T> py,
                Grid3<const T> pz, Grid3<const T> vx, Grid3<const T> vy,
                Grid3<const T> vz, FillBox fb) {
  CELL_LOOP_BEGIN(fb)
  T& r = rhs(i, j, k);
  r = r - (vx(i, j, k) * px(i, j, k) + vy(i, j, k) * py(i, j, k) +
           vz(i, j, k) * pz(i, j, k));
  CELL_LOOP_END
}

// Godunov |grad phi|^2 (lsm_level_set_evolution3d.f.in:209-227)
template <typename T>
__device__ __forceinline__ T godunov_sq(T vn, T xp, T yp, T zp, T xm, T ym,
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

// lsm_level_set_evolution3d.f.in:131-242 (array speed) / :248-350 (constant)
template <typename T, bool CONST_VN>
__global__ void __launch_bounds__(128)
k_add_normal(Grid3<T> rhs, Grid3<const T> xp, Grid3<const T> yp,
             Grid3<const T> zp, Grid3<const T> xm, Grid3<const T> ym,
             Grid3<const T> zm, Grid3<const T> vn, T vn_const, FillBox fb) {
  CELL_LOOP_BEGIN(fb)
  const T f = CONST_VN ? vn_const : vn(i, j, k);
  if (fabsT(f) >= Consts<T>::zero_tol) {
    const T s = godunov_sq(f, xp(i, j, k), yp(i, j, k), zp(i, j, k),
                           xm(i, j, k), ym(i, j, k), zm(i, j, k));
    T& r = rhs(i, j, k);
    r = r - f * sqrtT(s);
  }
  CELL_LOOP_END
}

// Godunov selection and smoothed-sign RHS of the reinitialization equation
// (lsm_reinitialization3d.f.in:158-199 and :218-256)
template <typename T>
__device__ __forceinline__ T reinit_rhs_cell(T phi_cur, T xp, T yp, T zp,
                                             T xm, T ym, T zm, T dx_sq,
                                             bool use_phi0) {
  const T z = T(0);
  T gp[3] = {xp, yp, zp}, gm[3] = {xm, ym, zm}, gs[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (phi_cur > z) {
      gp[d] = fmax2(-gp[d], z);
      gm[d] = fmax2(gm[d], z);
    } else {
      gp[d] = fmax2(gp[d], z);
      gm[d] = fmax2(-gm[d], z);
    }
    gs[d] = fmax2(gp[d], gm[d]);
  }
  if (fabsT(phi_cur) >= Consts<T>::zero_tol) {
    const T nsq = gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2];
    const T sgn = use_phi0 ? phi_cur / sqrtT(phi_cur * phi_cur + dx_sq)
                           : phi_cur / sqrtT(phi_cur * phi_cur + nsq * dx_sq);
    return sgn * (T(1) - sqrtT(nsq));
  }
  return z;
}

template <typename T>
__global__ void __launch_bounds__(128)
k_reinit_rhs(Grid3<T> rhs, Grid3<const T> phi, Grid3<const T> phi0,
             Grid3<const T> xp, Grid3<const T> yp, Grid3<const T> zp,
             Grid3<const T> xm, Grid3<const T> ym, Grid3<const T> zm,
             FillBox fb, T dx_sq, int use_phi0) {
  CELL_LOOP_BEGIN(fb)
  const bool u0 = (use_phi0 == 1);
  const T pc = u0 ? phi0(i, j, k) : phi(i, j, k);
  rhs(i, j, k) = reinit_rhs_cell(pc, xp(i, j, k), yp(i, j, k), zp(i, j, k),
                                 xm(i, j, k), ym(i, j, k), zm(i, j, k), dx_sq,
                                 u0);
  CELL_LOOP_END
}

// lsm_field_extension3d.f:118-151
template <typename T>
__global__ void __launch_bounds__(128)
k_field_ext(Grid3<T> rhs, Grid3<const T> phi, Grid3<const T> sx,
            Grid3<const T> sy, Grid3<const T> sz, Grid3<const T> nx,
            Grid3<const T> ny, Grid3<const T> nz, FillBox fb, T cutoff) {
  CELL_LOOP_BEGIN(fb)
  const T* q = phi.ptr(i, j, k);
  const T p = q[0];
  const T z = T(0);
  bool on;
  if (fabsT(p) > cutoff) {
    on = true;
  } else {
    on = (p * q[-1] > z) && (p * q[1] > z) && (p * q[-phi.sy] > z) &&
         (p * q[phi.sy] > z) && (p * q[-phi.sz] > z) && (p * q[phi.sz] > z);
  }
  rhs(i, j, k) = on ? -(nx(i, j, k) * sx(i, j, k) + ny(i, j, k) * sy(i, j, k) +
                        nz(i, j, k) * sz(i, j, k))
                    : z;
  CELL_LOOP_END
}

// lsm_geometry3d_fort.f.in:196-236
template <typename T>
__global__ void __launch_bounds__(128)
k_signed_normal(Grid3<T> nx, Grid3<T> ny, Grid3<T> nz, Grid3<const T> px,
                Grid3<const T> py, Grid3<const T> pz, Grid3<const T> phi,
                FillBox fb, T dx_sq) {
  CELL_LOOP_BEGIN(fb)
  const T pc = phi(i, j, k);
  const T gx = px(i, j, k), gy = py(i, j, k), gz = pz(i, j, k);
  T a = T(0), b = T(0), c = T(0);
  if (fabsT(pc) > Consts<T>::zero_tol) {
    const T nsq = gx * gx + gy * gy + gz * gz;
    if (nsq >= Consts<T>::zero_tol) {
      const T sgn = pc / sqrtT(pc * pc + nsq * dx_sq);
      const T inv = T(1) / sqrtT(nsq);
      a = sgn * gx * inv;
      b = sgn * gy * inv;
      c = sgn * gz * inv;
    } else {
      a = T(1);
    }
  }
  nx(i, j, k) = a;
  ny(i, j, k) = b;
  nz(i, j, k) = c;
  CELL_LOOP_END
}

// TVD Runge-Kutta updates (lsm_tvd_runge_kutta3d.f:78, :240, :403, :490)
template <typename T>
__device__ __forceinline__ T rk_update(int kind, T uc, T us, T r, T dt) {
  switch (kind) {
    case 22: return T(0.5) * (uc + us + dt * r);
    case 32: return T(0.75) * uc + T(0.25) * (us + dt * r);
    case 33: return (T(1) / T(3)) * uc + (T(2) / T(3)) * (us + dt * r);
    default: return uc + dt * r;
  }
}

template <typename T>
__global__ void __launch_bounds__(128)
k_rk(Grid3<T> out, Grid3<const T> us, Grid3<const T> uc, Grid3<const T> rhs,
     FillBox fb, int kind, T dt, const double* dt_dev, unsigned sr_seed) {
  const T h = dt_dev ? (T)(*dt_dev) : dt;
  CELL_LOOP_BEGIN(fb)
  const T s = (kind == 1) ? T(0) : us(i, j, k);
  if (sizeof(T) == 4 && sr_seed != 0u) {
    // FP32 state with stochastic rounding (common.cuh): the update in FP64
    const double hd = dt_dev ? *dt_dev : (double)dt;
    const double v = rk_update<double>(kind, uc(i, j, k), s, rhs(i, j, k), hd);
    const unsigned o = (unsigned)(i + out.sy * j + out.sz * k);
    out(i, j, k) = (T)sr_float(v, sr_hash(o * 0x9e3779b9u ^ sr_seed));
  } else {
    out(i, j, k) = rk_update(kind, uc(i, j, k), s, rhs(i, j, k), h);
  }
  CELL_LOOP_END
}

// Boundary conditions: one thread per line normal to the face
// (lsm_boundary_conditions3d.f:46-170 linear, :352-463 copy)
template <typename T>
__global__ void k_bc(Grid3<T> phi, Box gb, FillBox fb, int face, int copy) {
  const int d = face / 2, upper = face % 2;
  const int a = (d == 0) ? 1 : 0;          // fastest tangential axis
  const int b = (d == 2) ? 1 : 2;          // slowest tangential axis
  const int na = gb.n[a], nb = gb.n[b];
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)na * nb) return;
  int c[3];
  c[a] = gb.lo[a] + (int)(t % na);
  c[b] = gb.lo[b] + (int)(t / na);
  const long s = phi.stride(d);
  if (!upper) {
    c[d] = fb.lo[d];
    T* e = phi.ptr(c[0], c[1], c[2]);
    const T e0 = e[0];
    const T slope = e0 - e[s];
    for (int n = gb.lo[d]; n <= fb.lo[d] - 1; n++) {
      const T dist = (T)(fb.lo[d] - n);
      e[(long)(n - fb.lo[d]) * s] = copy ? e0 : e0 + slope * dist;
    }
  } else {
    c[d] = fb.hi[d];
    T* e = phi.ptr(c[0], c[1], c[2]);
    const T e0 = e[0];
    const T slope = e0 - e[-s];
    for (int n = fb.hi[d] + 1; n <= gb.hi(d); n++) {
      const T dist = (T)(n - fb.hi[d]);
      e[(long)(n - fb.hi[d]) * s] = copy ? e0 : e0 + slope * dist;
    }
  }
}

// ---------------------------------------------------------------------------
// reductions: per-block maxima with the reference's "if (v > m) m = v"
// comparison (NaN never replaces the running value), then a one-block finish
// ---------------------------------------------------------------------------
constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 1184;   // 148 SMs x 8

__device__ __forceinline__ double gt_max(double m, double v) {
  return (v > m) ? v : m;
}

__device__ __forceinline__ double block_max(double m) {
  __shared__ double sm[kRedThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = gt_max(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) sm[w] = m;
  __syncthreads();
  if (w == 0) {
    m = (l < kRedThreads / 32) ? sm[l] : -1.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = gt_max(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  return m;
}

struct IbIter {
  FillBox ib;
  long n;
  __device__ void at(long t, int& i, int& j, int& k) const {
    const long nx = ib.n(0), ny = ib.n(1);
    i = ib.lo[0] + (int)(t % nx);
    const long r = t / nx;
    j = ib.lo[1] + (int)(r % ny);
    k = ib.lo[2] + (int)(r / ny);
  }
};

template <typename T>
__global__ void __launch_bounds__(kRedThreads)
k_red_maxnorm(Grid3<const T> f1, Grid3<const T> f2, IbIter it,
              double* partials) {
  double m = -1.0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < it.n;
       t += (long)gridDim.x * blockDim.x) {
    int i, j, k;
    it.at(t, i, j, k);
    const double d = (double)fabsT(f1(i, j, k) - f2(i, j, k));
    m = gt_max(m, d);
  }
  m = block_max(m);
  if (threadIdx.x == 0) partials[blockIdx.x] = m;
}

// lsm_utilities3d.f.in:299-312
template <typename T>
__global__ void __launch_bounds__(kRedThreads)
k_red_adv_dt(Grid3<const T> vx, Grid3<const T> vy, Grid3<const T> vz,
             IbIter it, T ix, T iy, T iz, double* partials) {
  double m = -1.0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < it.n;
       t += (long)gridDim.x * blockDim.x) {
    int i, j, k;
    it.at(t, i, j, k);
    const T u = fabsT(vx(i, j, k)) * ix + fabsT(vy(i, j, k)) * iy +
                fabsT(vz(i, j, k)) * iz;
    m = gt_max(m, (double)u);
  }
  m = block_max(m);
  if (threadIdx.x == 0) partials[blockIdx.x] = m;
}

// Hamiltonian speed of one cell (lsm_utilities3d.f.in:410-427)
template <typename T>
__device__ __forceinline__ T normal_H(T absF, T xp, T yp, T zp, T xm, T ym,
                                      T zm, T max_dx_sq, T ix, T iy, T iz) {
  const T cx = fmax2(fabsT(xp), fabsT(xm));
  const T cy = fmax2(fabsT(yp), fabsT(ym));
  const T cz = fmax2(fabsT(zp), fabsT(zm));
  const T ng = sqrtT(cx * cx + cy * cy + cz * cz + max_dx_sq);
  return absF / ng * (cx * ix + cy * iy + cz * iz);
}

template <typename T, bool CONST_VN>
__global__ void __launch_bounds__(kRedThreads)
k_red_normal_dt(Grid3<const T> vn, T vn_const, Grid3<const T> xp,
                Grid3<const T> yp, Grid3<const T> zp, Grid3<const T> xm,
                Grid3<const T> ym, Grid3<const T> zm, IbIter it, T ix, T iy,
                T iz, T max_dx_sq, double* partials) {
  double m = -1.0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < it.n;
       t += (long)gridDim.x * blockDim.x) {
    int i, j, k;
    it.at(t, i, j, k);
    const T f = CONST_VN ? fabsT(vn_const) : fabsT(vn(i, j, k));
    const T h = normal_H(f, xp(i, j, k), yp(i, j, k), zp(i, j, k),
                         xm(i, j, k), ym(i, j, k), zm(i, j, k), max_dx_sq, ix,
                         iy, iz);
    m = gt_max(m, (double)h);
  }
  m = block_max(m);
  if (threadIdx.x == 0) partials[blockIdx.x] = m;
}

// mode 0: result = max (seeded with ``first`` when has_first), mode 1:
// result = cfl / (max + tiny)
__global__ void __launch_bounds__(kRedThreads)
k_red_finish(const double* partials, int np, int mode, double cfl,
             double tiny, const void* first_a, const void* first_b,
             int prec, double* result) {
  double m = -1.0;
  for (int t = threadIdx.x; t < np; t += blockDim.x) m = gt_max(m, partials[t]);
  m = block_max(m);
  if (threadIdx.x == 0) {
    if (mode == 0) {
      // lsm_utilities3d.f.in:57-70: the running max starts at the first cell
      double m0;
      if (prec == 8)
        m0 = fabs(*(const double*)first_a - *(const double*)first_b);
      else
        m0 = (double)fabsf(*(const float*)first_a - *(const float*)first_b);
      *result = gt_max(m0, m);
    } else {
      *result = cfl / (m + tiny);
    }
  }
}

template <typename T>
Grid3<T> G(void* p, const Box& b) { return make_grid((T*)p, b); }
template <typename T>
Grid3<const T> GC(const void* p, const Box& b) {
  return make_grid((const T*)p, b);
}

template <typename T>
cudaError_t hj_pm_t(int scheme, void* const op[3], const Box& gp,
                    void* const om[3], const Box& gm, const void* phi,
                    const Box& gphi, const FillBox& fb, const double inv[3],
                    cudaStream_t st) {
  dim3 grid = cell_grid(fb), blk(kBX, kBY, 1);
  auto args = [&](auto kern) {
    kern<<<grid, blk, 0, st>>>(G<T>(op[0], gp), G<T>(op[1], gp), G<T>(op[2], gp),
                               G<T>(om[0], gm), G<T>(om[1], gm), G<T>(om[2], gm),
                               GC<T>(phi, gphi), fb, (T)inv[0], (T)inv[1],
                               (T)inv[2]);
  };
  switch (scheme) {
    case kENO1: args(k_hj_plus_minus<kENO1, T>); break;
    case kENO2: args(k_hj_plus_minus<kENO2, T>); break;
    case kENO3: args(k_hj_plus_minus<kENO3, T>); break;
    default: args(k_hj_plus_minus<kWENO5, T>); break;
  }
  return post_launch();
}

template <typename T>
cudaError_t hj_up_t(int scheme, void* const o[3], const Box& go,
                    const void* phi, const Box& gphi, const void* const v[3],
                    const Box& gv, const FillBox& fb, const double inv[3],
                    cudaStream_t st) {
  dim3 grid = cell_grid(fb), blk(kBX, kBY, 1);
  auto args = [&](auto kern) {
    kern<<<grid, blk, 0, st>>>(G<T>(o[0], go), G<T>(o[1], go), G<T>(o[2], go),
                               GC<T>(phi, gphi), GC<T>(v[0], gv),
                               GC<T>(v[1], gv), GC<T>(v[2], gv), fb,
                               (T)inv[0], (T)inv[1], (T)inv[2]);
  };
  switch (scheme) {
    case kENO1: args(k_hj_upwind<kENO1, T>); break;
    case kENO2: args(k_hj_upwind<kENO2, T>); break;
    case kENO3: args(k_hj_upwind<kENO3, T>); break;
    default: args(k_hj_upwind<kWENO5, T>); break;
  }
  return post_launch();
}

inline int red_blocks(long n) {
  long b = (n + kRedThreads - 1) / kRedThreads;
  if (b < 1) b = 1;
  if (b > kRedMaxBlocks) b = kRedMaxBlocks;
  return (int)b;
}

}  // namespace

#define DISPATCH_PREC(prec, CALL) \
  ((prec) == 8 ? CALL(double) : CALL(float))

cudaError_t launch_hj_plus_minus(int scheme, int prec, void* const op[3],
                                 const Box& gp, void* const om[3],
                                 const Box& gm, const void* phi,
                                 const Box& gphi, const FillBox& fb,
                                 const double inv[3], cudaStream_t st) {
#define C(T) hj_pm_t<T>(scheme, op, gp, om, gm, phi, gphi, fb, inv, st)
  return DISPATCH_PREC(prec, C);
#undef C
}

cudaError_t launch_hj_upwind(int scheme, int prec, void* const out[3],
                             const Box& gout, const void* phi, const Box& gphi,
                             const void* const vel[3], const Box& gvel,
                             const FillBox& fb, const double inv[3],
                             cudaStream_t st) {
#define C(T) hj_up_t<T>(scheme, out, gout, phi, gphi, vel, gvel, fb, inv, st)
  return DISPATCH_PREC(prec, C);
#undef C
}

cudaError_t launch_fill(int prec, void* p, long count, double value,
                        cudaStream_t st) {
  int blocks = (int)((count + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  if (prec == 8) k_fill<double><<<blocks, 256, 0, st>>>((double*)p, count, value);
  else k_fill<float><<<blocks, 256, 0, st>>>((float*)p, count, (float)value);
  return post_launch();
}

cudaError_t launch_add_advection(int prec, void* rhs, const Box& grhs,
                                 const void* const g[3], const Box& gg,
                                 const void* const v[3], const Box& gv,
                                 const FillBox& fb, cudaStream_t st) {
  dim3 grid = cell_grid(fb), blk(kBX, kBY, 1);
#define C(T)                                                                  \
  (k_add_advection<T><<<grid, blk, 0, st>>>(                                  \
       G<T>(rhs, grhs), GC<T>(g[0], gg), GC<T>(g[1], gg), GC<T>(g[2], gg),    \
       GC<T>(v[0], gv), GC<T>(v[1], gv), GC<T>(v[2], gv), fb),                \
   0)
  DISPATCH_PREC(prec, C);
#undef C
  return post_launch();
}

cudaError_t launch_add_normal(int prec, void* rhs, const Box& grhs,
                              const void* const gp[3], const Box& gplus,
                              const void* const gm[3], const Box& gminus,
                              const void* vel_n, const Box& gvel,
                              double vn_const, const FillBox& fb,
                              cudaStream_t st) {
  dim3 grid = cell_grid(fb), blk(kBX, kBY, 1);
#define C(T)                                                                   \
  (vel_n ? (k_add_normal<T, false><<<grid, blk, 0, st>>>(                      \
                G<T>(rhs, grhs), GC<T>(gp[0], gplus), GC<T>(gp[1], gplus),     \
                GC<T>(gp[2], gplus), GC<T>(gm[0], gminus),                     \
                GC<T>(gm[1], gminus), GC<T>(gm[2], gminus),                    \
                GC<T>(vel_n, gvel), (T)0, fb),                                 \
            0)                                                                 \
         : (k_add_normal<T, true><<<grid, blk, 0, st>>>(                       \
                G<T>(rhs, grhs), GC<T>(gp[0], gplus), GC<T>(gp[1], gplus),     \
                GC<T>(gp[2], gplus), GC<T>(gm[0], gminus),                     \
                GC<T>(gm[1], gminus), GC<T>(gm[2], gminus),                    \
                GC<T>(gp[0], gplus), (T)vn_const, fb),                         \
            0))
  DISPATCH_PREC(prec, C);
#undef C
  return post_launch();
}

cudaError_t launch_reinit_rhs(int prec, void* rhs, const Box& grhs,
                              const void* phi, const Box& gphi,
                              const void* phi0, const Box& gphi0,
                              const void* const gp[3], const Box& gplus,
                              const void* const gm[3], const Box& gminus,
                              const FillBox& fb, double dx_sq, int use_phi0,
                              cudaStream_t st) {
  dim3 grid = cell_grid(fb), blk(kBX, kBY, 1);
#define C(T)                                                                  \
  (k_reinit_rhs<T><<<grid, blk, 0, st>>>(                                     \
       G<T>(rhs, grhs), GC<T>(phi, gphi), GC<T>(phi0, gphi0),                 \
       GC<T>(gp[0], gplus), GC<T>(gp[1], gplus), GC<T>(gp[2], gplus),         \
       GC<T>(gm[0], gminus), GC<T>(gm[1], gminus), GC<T>(gm[2], gminus), fb,  \
       (T)dx_sq, use_phi0),                                                   \
   0)
  DISPATCH_PREC(prec, C);
#undef C
  return post_launch();
}

cudaError_t launch_field_ext_rhs(int prec, void* rhs, const Box& grhs,
                                 const void* phi, const Box& gphi,
                                 const void* const gs[3], const Box& ggs,
                                 const void* const nrm[3], const Box& gn,
                                 const FillBox& fb, double cutoff,
                                 cudaStream_t st) {
  dim3 grid = cell_grid(fb), blk(kBX, kBY, 1);
#define C(T)                                                                  \
  (k_field_ext<T><<<grid, blk, 0, st>>>(                                      \
       G<T>(rhs, grhs), GC<T>(phi, gphi), GC<T>(gs[0], ggs),                  \
       GC<T>(gs[1], ggs), GC<T>(gs[2], ggs), GC<T>(nrm[0], gn),               \
       GC<T>(nrm[1], gn), GC<T>(nrm[2], gn), fb, (T)cutoff),                  \
   0)
  DISPATCH_PREC(prec, C);
#undef C
  return post_launch();
}

cudaError_t launch_signed_normal(int prec, void* const nrm[3], const Box& gn,
                                 const void* const g[3], const Box& gg,
                                 const void* phi, const Box& gphi,
                                 const FillBox& fb, double dx_sq,
                                 cudaStream_t st) {
  dim3 grid = cell_grid(fb), blk(kBX, kBY, 1);
#define C(T)                                                                  \
  (k_signed_normal<T><<<grid, blk, 0, st>>>(                                  \
       G<T>(nrm[0], gn), G<T>(nrm[1], gn), G<T>(nrm[2], gn), GC<T>(g[0], gg), \
       GC<T>(g[1], gg), GC<T>(g[2], gg), GC<T>(phi, gphi), fb, (T)dx_sq),     \
   0)
  DISPATCH_PREC(prec, C);
#undef C
  return post_launch();
}

cudaError_t launch_rk(int prec, int kind, void* out, const Box& gout,
                      const void* us, const Box& gus, const void* uc,
                      const Box& guc, const void* rhs, const Box& grhs,
                      const FillBox& fb, double dt, const double* dt_dev,
                      cudaStream_t st, unsigned sr_seed) {
  dim3 grid = cell_grid(fb), blk(kBX, kBY, 1);
  const void* usp = us ? us : uc;
  const Box& gusb = us ? gus : guc;
#define C(T)                                                                  \
  (k_rk<T><<<grid, blk, 0, st>>>(G<T>(out, gout), GC<T>(usp, gusb),           \
                                 GC<T>(uc, guc), GC<T>(rhs, grhs), fb, kind,  \
                                 (T)dt, dt_dev, sr_seed),                     \
   0)
  DISPATCH_PREC(prec, C);
#undef C
  return post_launch();
}

cudaError_t launch_bc(int prec, int copy, void* phi, const Box& gphi,
                      const FillBox& fb, int face, cudaStream_t st) {
  const int d = face / 2;
  const int a = (d == 0) ? 1 : 0, b = (d == 2) ? 1 : 2;
  const long lines = (long)gphi.n[a] * gphi.n[b];
  const int blocks = (int)((lines + 127) / 128);
  if (prec == 8)
    k_bc<double><<<blocks, 128, 0, st>>>(G<double>(phi, gphi), gphi, fb, face, copy);
  else
    k_bc<float><<<blocks, 128, 0, st>>>(G<float>(phi, gphi), gphi, fb, face, copy);
  return post_launch();
}

int reduce_partials_needed(const FillBox& ib) {
  return red_blocks(ib.count());
}

static cudaError_t finish(const double* partials, int np, int mode, double cfl,
                          double tiny, const void* fa, const void* fbp,
                          int prec, double* result, cudaStream_t st) {
  k_red_finish<<<1, kRedThreads, 0, st>>>(partials, np, mode, cfl, tiny, fa,
                                          fbp, prec, result);
  return post_launch();
}

cudaError_t launch_max_norm_diff(int prec, const void* f1, const Box& g1,
                                 const void* f2, const Box& g2,
                                 const FillBox& ib, double* partials,
                                 double* result_dev, cudaStream_t st) {
  IbIter it{ib, ib.count()};
  const int nb = red_blocks(it.n);
  const void *fa, *fbp;
  if (prec == 8) {
    Grid3<const double> a = GC<double>(f1, g1), b = GC<double>(f2, g2);
    k_red_maxnorm<double><<<nb, kRedThreads, 0, st>>>(a, b, it, partials);
    fa = a.ptr(ib.lo[0], ib.lo[1], ib.lo[2]);
    fbp = b.ptr(ib.lo[0], ib.lo[1], ib.lo[2]);
  } else {
    Grid3<const float> a = GC<float>(f1, g1), b = GC<float>(f2, g2);
    k_red_maxnorm<float><<<nb, kRedThreads, 0, st>>>(a, b, it, partials);
    fa = a.ptr(ib.lo[0], ib.lo[1], ib.lo[2]);
    fbp = b.ptr(ib.lo[0], ib.lo[1], ib.lo[2]);
  }
  cudaError_t e = post_launch();
  if (e != cudaSuccess) return e;
  return finish(partials, nb, 0, 0.0, 0.0, fa, fbp, prec, result_dev, st);
}

cudaError_t launch_stable_advection_dt(int prec, const void* const v[3],
                                       const Box& gv, const FillBox& ib,
                                       const double inv[3], double cfl,
                                       double* partials, double* result_dev,
                                       cudaStream_t st) {
  IbIter it{ib, ib.count()};
  const int nb = red_blocks(it.n);
#define C(T)                                                                  \
  (k_red_adv_dt<T><<<nb, kRedThreads, 0, st>>>(                               \
       GC<T>(v[0], gv), GC<T>(v[1], gv), GC<T>(v[2], gv), it, (T)inv[0],      \
       (T)inv[1], (T)inv[2], partials),                                       \
   0)
  DISPATCH_PREC(prec, C);
#undef C
  cudaError_t e = post_launch();
  if (e != cudaSuccess) return e;
  const double tiny = prec == 8 ? Consts<double>::tiny : (double)Consts<float>::tiny;
  return finish(partials, nb, 1, cfl, tiny, nullptr, nullptr, prec, result_dev, st);
}

cudaError_t launch_stable_normal_dt(int prec, const void* vel_n,
                                    const Box& gvel, double vn_const,
                                    const void* const gp[3], const Box& gplus,
                                    const void* const gm[3], const Box& gminus,
                                    const FillBox& ib, const double inv[3],
                                    double max_dx_sq, double cfl,
                                    double* partials, double* result_dev,
                                    cudaStream_t st) {
  IbIter it{ib, ib.count()};
  const int nb = red_blocks(it.n);
#define C(T)                                                                   \
  (vel_n ? (k_red_normal_dt<T, false><<<nb, kRedThreads, 0, st>>>(             \
                GC<T>(vel_n, gvel), (T)0, GC<T>(gp[0], gplus),                 \
                GC<T>(gp[1], gplus), GC<T>(gp[2], gplus), GC<T>(gm[0], gminus),\
                GC<T>(gm[1], gminus), GC<T>(gm[2], gminus), it, (T)inv[0],     \
                (T)inv[1], (T)inv[2], (T)max_dx_sq, partials),                 \
            0)                                                                 \
         : (k_red_normal_dt<T, true><<<nb, kRedThreads, 0, st>>>(              \
                GC<T>(gp[0], gplus), (T)vn_const, GC<T>(gp[0], gplus),         \
                GC<T>(gp[1], gplus), GC<T>(gp[2], gplus), GC<T>(gm[0], gminus),\
                GC<T>(gm[1], gminus), GC<T>(gm[2], gminus), it, (T)inv[0],     \
                (T)inv[1], (T)inv[2], (T)max_dx_sq, partials),                 \
            0))
  DISPATCH_PREC(prec, C);
#undef C
  cudaError_t e = post_launch();
  if (e != cudaSuccess) return e;
  const double tiny = prec == 8 ? Consts<double>::tiny : (double)Consts<float>::tiny;
  return finish(partials, nb, 1, cfl, tiny, nullptr, nullptr, prec, result_dev, st);
}

}  // namespace lsmgpu
