// distance.cu -- signed distance function on the GPU with the values of the
// reference's fast marching method (computeDistanceFunction3d,
// src/serial/lsm_FMM_field_extension.c, src/toolbox/fast_marching_method).
//
// The reference marches a heap.  The front (points on or next to the zero
// level set) is initialised and marked KNOWN first; then the trial point of
// smallest |d| is accepted, one at a time, and every acceptance recomputes
// the trial values of its neighbours from all KNOWN points around them
// (:1021-1119 first order, :1232-1381 second order).  A point's final value
// is therefore the update over
//   - all its front neighbours,
//   - the free neighbours accepted before it,
//   - at second order, the next point along an axis when it is a front
//     point or was accepted before the neighbour whose acceptance made the
//     last update.
// "Accepted before" is decided by acceptance time.  Mostly the heap accepts
// in order of |d|, but an acceptance can lower a trial neighbour's value
// below the key just popped (the second-order update is not monotone); the
// heap then pops that neighbour next.  So a point's time is the pair
// (e, s): e the largest key popped up to its acceptance, s = -1 when its
// own key is e, else its |d|.
// The GPU computes the march's result as the fixed point of these rules,
// without a heap:
//   1. the front is initialised cell by cell exactly as the reference does
//      (:397-668);
//   2. every other point starts unreached and is swept in place: each thread
//      walks a column in z (alternating up and down); a point takes its free
//      neighbours in order of time, each while it comes before the point's
//      own time given the ones taken so far, and stores its value and time
//      when either changes.  The sweeps stop when a batch of them changes
//      nothing.  A point depends only on points accepted before it, which
//      settle first;
//   3. points no front reaches keep the reference's default -1; points with
//      mask < 0 are outside the domain and hold LSMLIB_REAL_MAX.
// Built with --fmad=false so the update rounds as the reference's C does.
// Exact ties in time (equal keys) are broken by neighbour slot here and by
// heap position in the reference; only there can the results differ.
#include <cfloat>
#include <cmath>
#include <string>

#include "capi_common.h"
#include "launch.h"

using namespace lsmgpu;

namespace {

enum : unsigned char { kOutside = 0, kFront = 1, kFree = 2 };
constexpr double kZeroTol = 1.0e-11;   // LSMLIB_ZERO_TOL of the FP64 build

__device__ __forceinline__ long lin(int i, int j, int k, int nx, int ny) {
  return (long)i + (long)nx * ((long)j + (long)ny * k);
}

// FMM_initializeFront_FieldExtension3d_Order1 (lsm_FMM_field_extension.c:
// 397-668) for one point; the neighbours' phi is read whatever their mask
__global__ void k_fmm_front(double* d, double* e, unsigned char* st, const double* phi,
                            const double* mask, int nx, int ny, int nz, double dx,
                            double dy, double dz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const int n[3] = {nx, ny, nz};
  const double h[3] = {dx, dy, dz};
  for (int k = blockIdx.z; k < nz; k += gridDim.z) {
    const long o = lin(i, j, k, nx, ny);
    e[o] = INFINITY;
    if (mask && mask[o] < 0) {
      st[o] = kOutside;
      d[o] = DBL_MAX;
      continue;
    }
    const double pc = phi[o];
    if (fabs(pc) < kZeroTol) {           // on the interface
      st[o] = kFront;
      d[o] = pc > 0 ? kZeroTol : -kZeroTol;
      continue;
    }
    const int c[3] = {i, j, k};
    const long s[3] = {1L, (long)nx, (long)nx * ny};
    bool borders = false;
    double sum = 0;
    for (int dir = 0; dir < 3; dir++) {
      double dist_plus = DBL_MAX, dist_minus = DBL_MAX;
      if (c[dir] - 1 >= 0) {
        const double pm = phi[o - s[dir]];
        if (pm * pc <= 0) {
          dist_minus = pc / (pc - pm);
          dist_minus *= h[dir];
        }
      }
      if (c[dir] + 1 < n[dir]) {
        const double pp = phi[o + s[dir]];
        if (pp * pc <= 0) {
          dist_plus = pc / (pc - pp);
          dist_plus *= h[dir];
        }
      }
      if (dist_plus < DBL_MAX || dist_minus < DBL_MAX) {
        borders = true;
        const double dd = dist_plus < dist_minus ? dist_plus : dist_minus;
        sum += 1 / dd / dd;
      }
    }
    if (borders) {
      st[o] = kFront;
      d[o] = pc > 0 ? sqrt(1.0 / sum) : -sqrt(1.0 / sum);
    } else {
      st[o] = kFree;
      d[o] = pc > 0 ? INFINITY : -INFINITY;
    }
  }
}

// a neighbour that has a value (front or reached, inside the domain)
__device__ __forceinline__ bool known(const double* d, const unsigned char* st, long o) {
  return st[o] != kOutside && fabs(d[o]) <= DBL_MAX;
}

// Acceptance time of a free point in the reference's march, as the pair
// (e, s): e is the largest key popped from the heap up to and including the
// point's own acceptance, s is -1 for a point accepted with that key and |d|
// for a point whose value an acceptance lowered below e (the heap pops it,
// and the other lowered points in order of |d|, before any larger key).
// Front points are KNOWN before every free point.
__device__ __forceinline__ double time_s(double v, double e) {
  const double a = fabs(v);
  return a < e ? a : -1.0;
}
__device__ __forceinline__ bool before(double ea, double sa, double eb, double sb) {
  return ea < eb || (ea == eb && sa < sb);
}

// The neighbours of one point, by slot 2*axis + (plus side): the immediate
// neighbour (value v1, time e1) and, at second order, the next one in that
// direction (v2, e2).
struct Stencil {
  double v1[6], e1[6], v2[6], e2[6];
  unsigned char has1, front1, has2, front2;  // bit per slot
};

// The reference's trial update (:1021-1119 first order, :1232-1381 second
// order) over the immediate neighbours in ``incl`` (bit per slot).  Per axis
// the minus neighbour is taken when included and replaced by the plus one
// when its |d| is strictly smaller.  At second order the next point in the
// chosen direction counts when it was KNOWN at the update -- a front point,
// or a free point accepted before the neighbour whose acceptance made the
// update (time (te, ts); -inf in the front phase) -- and its |d| is not
// above the neighbour's.  Coefficients accumulate over x, y, z; returns
// false when the discriminant is negative (the reference then keeps the
// point's previous value).
template <int ORDER>
__device__ __forceinline__ bool fmm_quad(const Stencil& n, int incl, double te, double ts,
                                         const double i2[3], double& out) {
  double A = 0, B = 0, C = 0;
#pragma unroll
  for (int dir = 0; dir < 3; dir++) {
    double u1 = DBL_MAX, u2 = DBL_MAX;
    int sw = 0;
#pragma unroll
    for (int side = 0; side < 2; side++) {
      const int q = 2 * dir + side;
      if (!(incl & (1 << q))) continue;
      if (side == 1 && !(fabs(n.v1[q]) < fabs(u1))) continue;
      u1 = n.v1[q];
      u2 = DBL_MAX;
      sw = 0;
      if (ORDER == 2 && (n.has2 & (1 << q)) &&
          ((n.front2 & (1 << q)) || before(n.e2[q], time_s(n.v2[q], n.e2[q]), te, ts)) &&
          fabs(n.v2[q]) <= fabs(u1)) {
        u2 = n.v2[q];
        sw = 1;
      }
    }
    if (!(u1 < DBL_MAX)) continue;
    const double inv = i2[dir];
    if (ORDER == 1) {
      A += inv;
      B += inv * u1;
      C += inv * u1 * u1;
    } else {
      const double s = 1.0 + 0.5 * sw;
      const double contrib = sw == 1 ? 2.0 * u1 - 0.5 * u2 : u1;
      A += inv * s * s;
      B += inv * s * contrib;
      C += inv * contrib * contrib;
    }
  }
  B *= -2.0;
  C -= 1.0;
  const double disc = B * B - 4.0 * A * C;
  if (!(disc >= 0)) return false;
  if (B == 0) out = 0;
  else if (B < kZeroTol) out = 0.5 * (-B + sqrt(disc)) / A;
  else out = 0.5 * (-B - sqrt(disc)) / A;
  return true;
}

// The value and acceptance time of free point o from its neighbours' current
// values and times: the reference's last trial update.  Every front point is
// KNOWN before the march starts (FMM_Core.c:203-243), so the front
// neighbours are always in the update.  The free neighbours are taken in
// order of acceptance time; each is in the update when the heap accepted it
// while this point was still a trial point, i.e. before this point's time as
// given by the neighbours taken so far.  A negative discriminant keeps the
// previous value, -1 (the reference's default) when there is none.
template <int ORDER>
__device__ __forceinline__ void fmm_point(const double* d, const double* e,
                                          const unsigned char* st, long o, const int c[3],
                                          const int n[3], const long s[3], const double i2[3],
                                          double& val, double& ev, bool& any_known) {
  Stencil nb;
  nb.has1 = nb.front1 = nb.has2 = nb.front2 = 0;
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int dir = q >> 1;
    const int sg = (q & 1) ? 1 : -1;
    nb.v1[q] = nb.v2[q] = DBL_MAX;
    nb.e1[q] = nb.e2[q] = INFINITY;
    const int c1 = c[dir] + sg;
    if (c1 < 0 || c1 >= n[dir]) continue;
    const long o1 = o + sg * s[dir];
    if (!known(d, st, o1)) continue;
    nb.v1[q] = d[o1];
    nb.e1[q] = e[o1];
    nb.has1 |= 1 << q;
    if (st[o1] == kFront) nb.front1 |= 1 << q;
    if (ORDER == 2) {
      const int c2 = c1 + sg;
      if (c2 < 0 || c2 >= n[dir]) continue;
      const long o2 = o1 + sg * s[dir];
      if (!known(d, st, o2)) continue;
      nb.v2[q] = d[o2];
      nb.e2[q] = e[o2];
      nb.has2 |= 1 << q;
      if (st[o2] == kFront) nb.front2 |= 1 << q;
    }
  }
  any_known = nb.has1 != 0;
  if (!any_known) return;
  int incl = nb.front1;
  bool have = incl != 0;
  val = -1.0;
  double elast = -INFINITY;             // e of the last free neighbour taken
  double te = -INFINITY, ts = -1.0;     // its time (the front phase before all)
  if (have) {
    double t;
    if (fmm_quad<ORDER>(nb, incl, te, ts, i2, t)) val = t;
  }
  for (int rem = nb.has1 & ~nb.front1; rem;) {
    // the earliest remaining free neighbour (ties by slot)
    int best = 0;
    double be = INFINITY, bs = INFINITY;
#pragma unroll
    for (int q = 5; q >= 0; q--) {
      if (!(rem & (1 << q))) continue;
      const double eq = nb.e1[q], sq = time_s(nb.v1[q], nb.e1[q]);
      if (!before(be, bs, eq, sq)) {
        best = q;
        be = eq;
        bs = sq;
      }
    }
    rem &= ~(1 << best);
    if (have) {
      const double a = fabs(val);
      if (!before(be, bs, a > elast ? a : elast, a < elast ? a : -1.0)) break;
    }
    incl |= 1 << best;
    elast = te = be;
    ts = bs;
    double t;
    if (fmm_quad<ORDER>(nb, incl, te, ts, i2, t)) val = t;
    have = true;
  }
  const double a = fabs(val);
  ev = a > elast ? a : elast;
}

// One sweep over the free points, columns walked up (up != 0) or down in z;
// a point's value and time are stored when either changes.
template <int ORDER>
__global__ void k_fmm_sweep(double* d, double* e, const unsigned char* st, int nx, int ny,
                            int nz, double i2x, double i2y, double i2z, int up, int* changed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const double i2[3] = {i2x, i2y, i2z};
  const int n[3] = {nx, ny, nz};
  const long s[3] = {1L, (long)nx, (long)nx * ny};
  bool any = false;
  for (int kk = 0; kk < nz; kk++) {
    const int k = up ? kk : nz - 1 - kk;
    const long o = lin(i, j, k, nx, ny);
    if (st[o] != kFree) continue;
    const int c[3] = {i, j, k};
    double val, ev;
    bool known_nb;
    fmm_point<ORDER>(d, e, st, o, c, n, s, i2, val, ev, known_nb);
    if (!known_nb) continue;
    if (val != d[o] || ev != e[o]) {
      d[o] = val;
      e[o] = ev;
      any = true;
    }
  }
  if (any) *changed = 1;
}

// free points no front reached: the reference's default value -1
__global__ void k_fmm_unreached(double* d, const unsigned char* st, long n) {
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n;
       o += (long)gridDim.x * blockDim.x)
    if (st[o] == kFree && !(fabs(d[o]) <= DBL_MAX)) d[o] = -1.0;
}

int distance3d(double* distance, const double* phi, const double* mask, int order,
               const int* grid_dims, const double* dx, int* sweeps_out, const char* R) {
  clear_error();
  if (!distance || !phi || !grid_dims || !dx) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  if (order != 1 && order != 2) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": order is 1 or 2");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  const int nx = grid_dims[0], ny = grid_dims[1], nz = grid_dims[2];
  if (nx < 1 || ny < 1 || nz < 1) {
    set_error(LSMGPU_ERR_INVALID_BOX, std::string(R) + ": empty grid");
    return LSMGPU_ERR_INVALID_BOX;
  }
  if (!(dx[0] > 0) || !(dx[1] > 0) || !(dx[2] > 0)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": dx must be positive");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  const long n = (long)nx * ny * nz;
  cudaStream_t st = cur_stream();
  Staging s(st);
  const Box b{{0, 0, 0}, {nx, ny, nz}};
  double* dd = (double*)s.add(distance, b, 8, kOut, "distance_function", R);
  const double* dp = dd ? (const double*)s.add(phi, b, 8, kIn, "phi", R) : nullptr;
  const double* dm = nullptr;
  if (dp && mask) dm = (const double*)s.add(mask, b, 8, kIn, "mask", R);
  if (!dd || !dp || (mask && !dm)) return lsmgpu_peek_last_error();
  unsigned char* status = nullptr;
  double* etime = nullptr;
  int* changed = nullptr;
  int h_changed = 0;
  bool ok = cuda_ok(cudaMallocAsync((void**)&status, (size_t)n, st), R) &&
            cuda_ok(cudaMallocAsync((void**)&etime, (size_t)n * sizeof(double), st), R) &&
            cuda_ok(cudaMallocAsync((void**)&changed, sizeof(int), st), R);
  const dim3 blk(32, 4, 1);
  const dim3 grid2((nx + 31) / 32, (ny + 3) / 4, 1);
  const dim3 grid3((nx + 31) / 32, (ny + 3) / 4, nz < 65535 ? nz : 65535);
  if (ok) {
    k_fmm_front<<<grid3, blk, 0, st>>>(dd, etime, status, dp, dm, nx, ny, nz, dx[0], dx[1], dx[2]);
    ++launch_counter();
    ok = cuda_ok(cudaGetLastError(), R);
  }
  // 1/dx, squared (:1077-1078)
  double i2[3];
  for (int q = 0; q < 3; q++) {
    i2[q] = 1 / dx[q];
    i2[q] *= i2[q];
  }
  const int batch = 8;
  const long max_sweeps = 16L * (nx + ny + nz) + 256;
  long sweeps = 0;
  while (ok) {
    ok = cuda_ok(cudaMemsetAsync(changed, 0, sizeof(int), st), R);
    for (int q = 0; ok && q < batch; q++, sweeps++) {
      if (order == 1)
        k_fmm_sweep<1><<<grid2, blk, 0, st>>>(dd, etime, status, nx, ny, nz, i2[0], i2[1], i2[2],
                                              (int)(sweeps & 1) ^ 1, changed);
      else
        k_fmm_sweep<2><<<grid2, blk, 0, st>>>(dd, etime, status, nx, ny, nz, i2[0], i2[1], i2[2],
                                              (int)(sweeps & 1) ^ 1, changed);
      ++launch_counter();
    }
    ok = ok && cuda_ok(cudaGetLastError(), R) &&
         cuda_ok(cudaMemcpyAsync(&h_changed, changed, sizeof(int), cudaMemcpyDeviceToHost,
                                 st), R) &&
         cuda_ok(cudaStreamSynchronize(st), R);
    if (!ok || !h_changed) break;
    if (sweeps >= max_sweeps) {
      // the fixed point is reached well within this bound (about one sweep
      // per cell of the longest upwind path); it guards against inputs
      // without one
      set_error(LSMGPU_ERR_INVALID_VALUE,
                std::string(R) + ": no convergence (NaN in phi or dx?)");
      ok = false;
    }
  }
  if (ok) {
    const long nb = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
    k_fmm_unreached<<<(int)nb, 256, 0, st>>>(dd, status, n);
    ++launch_counter();
    ok = cuda_ok(cudaGetLastError(), R);
  }
  if (status) cudaFreeAsync(status, st);
  if (etime) cudaFreeAsync(etime, st);
  if (changed) cudaFreeAsync(changed, st);
  if (sweeps_out) *sweeps_out = (int)sweeps;
  if (!ok) return lsmgpu_peek_last_error() ? lsmgpu_peek_last_error() : LSMGPU_ERR_CUDA;
  return s.finish(R) ? LSMGPU_SUCCESS : LSMGPU_ERR_CUDA;
}

}  // namespace

extern "C" {

// lsm_fast_marching_method.h:386-392: 0 on success, 2 for an order other
// than 1 or 2 (LSM_FMM_ERR_INVALID_SPATIAL_DISCRETIZATION_ORDER), -1 for any
// other failure (the lsmgpu error is recorded)
int computeDistanceFunction3d(double* distance_function, double* phi, double* mask,
                              int spatial_discretization_order, int* grid_dims,
                              double* dx) {
  if (spatial_discretization_order != 1 && spatial_discretization_order != 2) return 2;
  const int rc = distance3d(distance_function, phi, mask, spatial_discretization_order,
                            grid_dims, dx, nullptr, "computeDistanceFunction3d");
  return rc == LSMGPU_SUCCESS ? 0 : -1;
}

int lsmgpu_distance_function3d(double* distance_function, const double* phi,
                               const double* mask, int order, const int* grid_dims,
                               const double* dx, int* sweeps) {
  return distance3d(distance_function, phi, mask, order, grid_dims, dx, sweeps,
                    "lsmgpu_distance_function3d");
}

}  // extern "C"
