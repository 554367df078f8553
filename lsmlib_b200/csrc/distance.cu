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
// "Accepted before" is decided by acceptance time (Time3 below): mostly the
// heap accepts in order of |d|, but an acceptance can lower a trial
// neighbour's value below the key just popped (the second-order update is
// not monotone), and the heap then pops that neighbour next.
// The GPU computes the march's result as the fixed point of these rules,
// without a heap:
//   1. the front is initialised cell by cell exactly as the reference does
//      (:397-668);
//   2. every other point starts unreached; passes over a band of active
//      points (below) evaluate the rules until nothing changes;
//   3. points no front reaches keep the reference's default -1; points with
//      mask < 0 are outside the domain and hold LSMLIB_REAL_MAX.
// Built with --fmad=false so the update rounds as the reference's C does.
// "Before" is the order of (acceptance time, linear point index): the time
// decides, and the index breaks exact ties.  Where no two keys tie this is
// the heap's pop order.  Where keys tie exactly (symmetric inputs, flat
// fronts, quantised data) the reference's binary heap pops the tied points in
// an order set by its whole history of insertions and removals, which no
// rule over a neighbourhood can reproduce; there the result is that of the
// same march popping ties by index.
#include <cfloat>
#include <climits>
#include <cmath>
#include <string>

#include "capi_common.h"
#include "launch.h"

using namespace lsmgpu;

namespace {

enum : unsigned char { kOutside = 0, kFront = 1, kFree = 2 };
constexpr double kZeroTol = 1.0e-11;   // LSMLIB_ZERO_TOL of the FP64 build

// Acceptance time of a free point, compared lexicographically.  A point the
// heap pops with the largest key so far (a "root") has time (|d|, -1, -1).
// A point an acceptance lowered below the keys already popped is popped
// right after its trigger (the last neighbour accepted before it), ahead of
// every larger key: its time extends the trigger's by its own |d| at the
// first level where |d| exceeds the trigger's key -- (a, |d|, -1) under a
// root trigger, (a, b, |d|) when it drops below a lowered trigger's key b.
// A time therefore always follows its trigger's.  Deeper lowering (below a
// third-level key) keeps the trigger's time; it has not been seen in
// practice.
struct Time3 {
  double a, b, c;
};

__device__ __forceinline__ bool tless(const Time3& x, const Time3& y) {
  return x.a < y.a || (x.a == y.a && (x.b < y.b || (x.b == y.b && x.c < y.c)));
}

__device__ __forceinline__ bool tequal(const Time3& x, const Time3& y) {
  return x.a == y.a && x.b == y.b && x.c == y.c;
}

// point x (time tx, linear index ix) is accepted before point y: by time,
// exact ties by index
__device__ __forceinline__ bool kless(const Time3& tx, long ix, const Time3& ty, long iy) {
  if (tless(tx, ty)) return true;
  if (tless(ty, tx)) return false;
  return ix < iy;
}

// linear index of the k-th point (k = 1, 2) from o in slot q's direction
__device__ __forceinline__ long nb_index(long o, const long s[3], int q, int k) {
  return o + ((q & 1) ? k : -k) * s[q >> 1];
}

// the time of a point with key ``a`` whose trigger has time ``x`` (no free
// trigger: a root)
__device__ __forceinline__ Time3 tafter(const Time3& x, double a, bool has_trigger) {
  if (!has_trigger || a > x.a) return Time3{a, -1.0, -1.0};
  if (x.b < 0 || a > x.b) return Time3{x.a, a, -1.0};
  if (x.c < 0 || a > x.c) return Time3{x.a, x.b, a};
  return x;
}

// Extension fields carried by one solve (computeExtensionFields3d): output
// fields, their source fields, the optional extension mask.
constexpr int kMaxFields = 8;
struct ExtSet {
  double* ext[kMaxFields];
  const double* src[kMaxFields];
  const double* emask;
  int nf;
};

// FMM_initializeFront_FieldExtension3d_Order1 (lsm_FMM_field_extension.c:
// 397-668) for one point; the neighbours' phi is read whatever their mask.
// Extension fields: every value starts at -1 (LSMLIB_REAL_MAX outside the
// mask); on the interface the source value; next to it the average over
// the axes of the source interpolated linearly to the nearer crossing (or
// taken from one side where the extension mask is < 0), weights
// 1/d_axis^2 (:524-660).
__global__ void k_fmm_front(double* d, Time3* tm, unsigned char* st, const double* phi,
                            const double* mask, int nx, int ny, int nz, double dx,
                            double dy, double dz, ExtSet X) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const int n[3] = {nx, ny, nz};
  const double h[3] = {dx, dy, dz};
  for (int k = blockIdx.z; k < nz; k += gridDim.z) {
    const long o = (long)i + (long)nx * ((long)j + (long)ny * k);
    tm[o] = Time3{INFINITY, INFINITY, INFINITY};
    if (mask && mask[o] < 0) {
      st[o] = kOutside;
      d[o] = DBL_MAX;
      for (int k = 0; k < X.nf; k++) X.ext[k][o] = DBL_MAX;
      continue;
    }
    const double pc = phi[o];
    if (fabs(pc) < kZeroTol) {           // on the interface
      st[o] = kFront;
      d[o] = pc > 0 ? kZeroTol : -kZeroTol;
      for (int k = 0; k < X.nf; k++) X.ext[k][o] = X.src[k][o];
      continue;
    }
    const int c[3] = {i, j, k};
    const long s[3] = {1L, (long)nx, (long)nx * ny};
    bool borders = false;
    double sum = 0;
    double fsum[kMaxFields];
#pragma unroll
    for (int f = 0; f < kMaxFields; f++) fsum[f] = 0;
    for (int dir = 0; dir < 3; dir++) {
      double dist_plus = DBL_MAX, dist_minus = DBL_MAX;
      double frac_plus = 0, frac_minus = 0;
      if (c[dir] - 1 >= 0) {
        const double pm = phi[o - s[dir]];
        if (pm * pc <= 0) {
          dist_minus = pc / (pc - pm);
          frac_minus = dist_minus;
          dist_minus *= h[dir];
        }
      }
      if (c[dir] + 1 < n[dir]) {
        const double pp = phi[o + s[dir]];
        if (pp * pc <= 0) {
          dist_plus = pc / (pc - pp);
          frac_plus = dist_plus;
          dist_plus *= h[dir];
        }
      }
      if (dist_plus < DBL_MAX || dist_minus < DBL_MAX) {
        borders = true;
        const bool use_plus = dist_plus < dist_minus;
        const double dd = use_plus ? dist_plus : dist_minus;
        const double w = 1 / dd / dd;
        sum += w;
        const long on = use_plus ? o + s[dir] : o - s[dir];
        const double frac = use_plus ? frac_plus : frac_minus;
#pragma unroll
        for (int f = 0; f < kMaxFields; f++) {
          if (f >= X.nf) break;
          const double cur = X.src[f][o];
          double v;
          if (X.emask && X.emask[o] < 0) v = X.src[f][on];
          else if (X.emask && X.emask[on] < 0) v = cur;
          else v = cur + frac * (X.src[f][on] - cur);
          fsum[f] += v * w;
        }
      }
    }
    if (borders) {
      st[o] = kFront;
      d[o] = pc > 0 ? sqrt(1.0 / sum) : -sqrt(1.0 / sum);
#pragma unroll
      for (int f = 0; f < kMaxFields; f++)
        if (f < X.nf) X.ext[f][o] = fsum[f] / sum;
    } else {
      st[o] = kFree;
      d[o] = pc > 0 ? INFINITY : -INFINITY;
      for (int f = 0; f < X.nf; f++) X.ext[f][o] = -1.0;
    }
  }
}

// The Eikonal solver's data (solveEikonalEquation3d): the speed F and the
// input phi, whose values the points never updated keep.  speed == nullptr
// for the distance function.
struct Eik {
  const double* speed;
  const double* phi0;
};

// FMM_initializeFront_Eikonal3d (lsm_FMM_eikonal.c:259-312) and the domain
// marking before it (:214-246): points with mask < 0 or speed < 1e-11 are
// outside the domain and get LSMLIB_REAL_MAX; points with phi > -1e-11 are
// the front, KNOWN with their own values; the others start unreached.
__global__ void k_eik_front(double* d, Time3* tm, unsigned char* st, const double* phi0,
                            const double* speed, const double* mask, long n) {
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n;
       o += (long)gridDim.x * blockDim.x) {
    tm[o] = Time3{INFINITY, INFINITY, INFINITY};
    if ((mask && mask[o] < 0) || speed[o] < kZeroTol) {
      st[o] = kOutside;
      d[o] = DBL_MAX;
    } else if (phi0[o] > -kZeroTol) {
      st[o] = kFront;
      d[o] = phi0[o];
    } else {
      st[o] = kFree;
      d[o] = INFINITY;
    }
  }
}

// The neighbours of one point, by slot 2*axis + (plus side): the immediate
// neighbour (value v1, time t1) and, at second order, the next one in that
// direction (v2, t2).
struct Stencil {
  double v1[6], v2[6];
  Time3 t1[6], t2[6];
  unsigned char has1, front1, has2, front2;  // bit per slot
};

// The coefficients of the reference's trial update (:1021-1119 first order,
// :1232-1381 second order) over the immediate neighbours in ``incl`` (bit
// per slot), accumulated in its order and rounding.  Per axis the minus
// neighbour is taken when included and replaced by the plus one when its
// |d| is strictly smaller.  At second order the next point in the chosen
// direction counts when it was KNOWN at the update -- a front point, or a
// free point accepted before the trigger (time ``trig``, index ``itrig``;
// the front phase comes before every free point) -- and its |d| is not above
// the neighbour's.  ``cterm`` is what the constant term loses: 1 for the
// distance function, 1/F^2 for the Eikonal solver (lsm_FMM_eikonal.c:427,
// :621).  Returns the discriminant B^2 - 4AC.
template <int ORDER>
__device__ __forceinline__ double fmm_coeffs(const Stencil& n, int incl,
                                             const Time3& trig, long itrig, bool has_trigger,
                                             long o, const long s3[3], const double i2[3],
                                             double cterm, double& A, double& B) {
  double C = 0;
  A = 0;
  B = 0;
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
      if (ORDER == 2 && (n.has2 & (1 << q)) && fabs(n.v2[q]) <= fabs(u1) &&
          ((n.front2 & (1 << q)) ||
           (has_trigger && kless(n.t2[q], nb_index(o, s3, q, 2), trig, itrig)))) {
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
  C -= cterm;
  return B * B - 4.0 * A * C;
}

// The root the reference takes (disc >= 0), in its rounding: by the sign
// of B for the distance function (lsm_FMM_field_extension.c:1106-1117), the
// larger root for the Eikonal solver (lsm_FMM_eikonal.c:433-436).
template <bool EIK>
__device__ __forceinline__ double fmm_root(double A, double B, double disc) {
  if (EIK) return 0.5 * (-B + sqrt(disc)) / A;
  if (B == 0) return 0;
  if (B < kZeroTol) return 0.5 * (-B + sqrt(disc)) / A;
  return 0.5 * (-B - sqrt(disc)) / A;
}

// ---- the band solver ----------------------------------------------------------
// The threshold T on acceptance time (its first level) advances in steps; a
// point's value is stored only while its time is within T.  A point depends
// only on points with earlier times, so the points within T settle exactly
// and are never revised once T has moved past them: the work follows a thin
// band, as the march does, instead of relaxing the whole grid.  Each pass
// evaluates the points of the active list, one thread per point, from its
// neighbours' current values; a point whose value or time changed queues
// the points whose stencil reads it for the next pass.  A point whose time
// is above T keeps its time as a candidate and waits in a pending list;
// when a pass queues nothing, T moves to max(T + delta, smallest
// candidate) and the pending points it reaches are queued.  A pass is two
// kernels: k_fmm_pass evaluates every queued point from the values before
// the pass (and, after a threshold advance, moves the pending points the
// new T reaches to the next queue), k_fmm_apply stores the changes, queues
// their readers and runs the threshold control in its last block.

// the threshold advances by this many of the smallest spacing per step
constexpr double kDeltaCells = 2.0;

// The value and acceptance time of free point o from its neighbours' current
// values and times: the reference's last trial update.  Every front point is
// KNOWN before the march starts (FMM_Core.c:203-243), so the front
// neighbours are always in the update.  The free neighbours are taken in
// order of time; each is in the update when the heap accepted it while this
// point was still a trial point, i.e. before this point's time as given by
// the neighbours taken so far.  The set must also be consistent with the
// point's final time -- every neighbour in it accepted before the point --
// as it always is in a real march; when it is not (a transient state of the
// passes), the set is cut before the earliest offending neighbour and the
// update is taken again.  A negative discriminant keeps the previous value:
// -1 (the reference's default) when there is none, or for the Eikonal
// solver the point's input.  Neighbours off the grid
// are left out, as the reference's bounds checks do.
template <int ORDER, bool EIK>
__device__ __forceinline__ bool fmm_point(const double* d, const Time3* tm,
                                          const unsigned char* st, long o, const int c[3],
                                          const int n[3], const long s[3], const double i2[3],
                                          const Eik& E, Stencil& nb, double& val, Time3& tv,
                                          int& incl_out, Time3& trig_out, long& itrig_out,
                                          bool& trig_free_out) {
  // every load first, at in-range addresses (the point itself stands in
  // for a neighbour off the grid), so that they are in flight together
  unsigned char s1[6], s2[6];
  bool in1[6], in2[6];
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int dir = q >> 1;
    const int sg = (q & 1) ? 1 : -1;
    in1[q] = c[dir] + sg >= 0 && c[dir] + sg < n[dir];
    const long o1 = in1[q] ? o + sg * s[dir] : o;
    s1[q] = st[o1];
    nb.v1[q] = d[o1];
    nb.t1[q] = tm[o1];
    if (ORDER == 2) {
      in2[q] = in1[q] && c[dir] + 2 * sg >= 0 && c[dir] + 2 * sg < n[dir];
      const long o2 = in2[q] ? o + 2 * sg * s[dir] : o;
      s2[q] = st[o2];
      nb.v2[q] = d[o2];
      nb.t2[q] = tm[o2];
    }
  }
  nb.has1 = nb.front1 = nb.has2 = nb.front2 = 0;
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const bool k1 = in1[q] && s1[q] != kOutside && fabs(nb.v1[q]) <= DBL_MAX;
    if (!k1) {
      nb.v1[q] = DBL_MAX;
      nb.t1[q] = Time3{INFINITY, INFINITY, INFINITY};
      continue;
    }
    nb.has1 |= 1 << q;
    if (s1[q] == kFront) {
      nb.front1 |= 1 << q;
      nb.t1[q] = Time3{INFINITY, INFINITY, INFINITY};
    }
    if (ORDER == 2) {
      const bool k2 = in2[q] && s2[q] != kOutside && fabs(nb.v2[q]) <= DBL_MAX;
      if (!k2) {
        nb.v2[q] = DBL_MAX;
        continue;
      }
      nb.has2 |= 1 << q;
      if (s2[q] == kFront) nb.front2 |= 1 << q;
    }
  }
  if (!nb.has1) return false;
  const int free1 = nb.has1 & ~nb.front1;
  const double cterm = EIK ? 1 / E.speed[o] / E.speed[o] : 1.0;
  const double none = EIK ? E.phi0[o] : -1.0;   // the value without an update
  // only neighbours before this (time, index)
  Time3 cap{INFINITY, INFINITY, INFINITY};
  long icap = LONG_MAX;
  for (;;) {
    int incl = nb.front1;
    bool have = incl != 0, trig_free = false;
    Time3 trig{-INFINITY, -1.0, -1.0};
    long itrig = -1;
    double cur = none;
    if (have) {
      double A, B;
      const double disc =
          fmm_coeffs<ORDER>(nb, incl, trig, itrig, false, o, s, i2, cterm, A, B);
      if (disc >= 0) cur = fmm_root<EIK>(A, B, disc);
    }
    for (int rem = free1; rem;) {
      // the earliest remaining free neighbour
      int best = -1;
      Time3 bt{INFINITY, INFINITY, INFINITY};
      long ib = LONG_MAX;
#pragma unroll
      for (int q = 5; q >= 0; q--) {
        if (!(rem & (1 << q))) continue;
        const long iq = nb_index(o, s, q, 1);
        if (best < 0 || kless(nb.t1[q], iq, bt, ib)) {
          best = q;
          bt = nb.t1[q];
          ib = iq;
        }
      }
      rem &= ~(1 << best);
      if (!kless(bt, ib, cap, icap)) break;
      if (have && !kless(bt, ib, tafter(trig, fabs(cur), trig_free), o)) break;
      incl |= 1 << best;
      trig = bt;
      itrig = ib;
      trig_free = true;
      double A, B;
      const double disc =
          fmm_coeffs<ORDER>(nb, incl, trig, itrig, true, o, s, i2, cterm, A, B);
      if (disc >= 0) cur = fmm_root<EIK>(A, B, disc);
      have = true;
    }
    const Time3 t = tafter(trig, fabs(cur), trig_free);
    // the earliest neighbour in the set not accepted before the point
    bool bad = false;
    Time3 badt{INFINITY, INFINITY, INFINITY};
    long ibad = LONG_MAX;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      if (!(incl & free1 & (1 << q))) continue;
      const long iq = nb_index(o, s, q, 1);
      if (!kless(nb.t1[q], iq, t, o) && kless(nb.t1[q], iq, badt, ibad)) {
        bad = true;
        badt = nb.t1[q];
        ibad = iq;
      }
    }
    if (!bad) {
      val = cur;
      tv = t;
      incl_out = incl;
      trig_out = trig;
      itrig_out = itrig;
      trig_free_out = trig_free;
      return true;
    }
    cap = badt;
    icap = ibad;
  }
}

// The extension fields of the point's last trial update: over the axes in
// the update, the weighted average of the upwind neighbour's field with
// weights (dist - phi_upwind)/dx^2, or (1.5 dist - 2 phi_upwind1 +
// 0.5 phi_upwind2)/dx^2 where the second-order stencil is used
// (lsm_FMM_field_extension.c:1135-1168, :1400-1460); ``val`` is the
// update's distance (the previous one where the discriminant was
// negative).  Each field whose value changes is stored; returns whether any
// did.
template <int ORDER>
__device__ __forceinline__ bool fmm_ext(const Stencil& n, int incl, const Time3& trig,
                                        long itrig, bool has_trigger, double val,
                                        const double i2[3], const ExtSet& X, long o,
                                        const long s[3]) {
  double g[3];
  long a[3];
  bool used[3];
#pragma unroll
  for (int dir = 0; dir < 3; dir++) {
    double u1 = DBL_MAX, u2 = DBL_MAX;
    int sw = 0, side_used = -1;
#pragma unroll
    for (int side = 0; side < 2; side++) {
      const int q = 2 * dir + side;
      if (!(incl & (1 << q))) continue;
      if (side == 1 && !(fabs(n.v1[q]) < fabs(u1))) continue;
      u1 = n.v1[q];
      u2 = DBL_MAX;
      sw = 0;
      side_used = side;
      if (ORDER == 2 && (n.has2 & (1 << q)) && fabs(n.v2[q]) <= fabs(u1) &&
          ((n.front2 & (1 << q)) ||
           (has_trigger && kless(n.t2[q], nb_index(o, s, q, 2), trig, itrig)))) {
        u2 = n.v2[q];
        sw = 1;
      }
    }
    used[dir] = side_used >= 0;
    a[dir] = side_used == 1 ? o + s[dir] : o - s[dir];
    g[dir] = (ORDER == 2 && sw == 1) ? 1.5 * val - 2.0 * u1 + 0.5 * u2 : val - u1;
  }
  bool changed = false;
#pragma unroll
  for (int f = 0; f < kMaxFields; f++) {
    if (f >= X.nf) break;
    double num = 0, den = 0;
#pragma unroll
    for (int dir = 0; dir < 3; dir++) {
      if (!used[dir]) continue;
      num += i2[dir] * g[dir] * X.ext[f][a[dir]];
      den += i2[dir] * g[dir];
    }
    const double v = num / den;
    if (__double_as_longlong(v) != __double_as_longlong(X.ext[f][o])) {
      X.ext[f][o] = v;
      changed = true;
    }
  }
  return changed;
}

// Device state of the solve, read and advanced by the kernels so that the
// host only launches and, every few passes, looks at ``done``.
struct Ctrl {
  int pass;                  // passes run so far
  int count[2];              // lengths of the two active lists (by pass parity)
  int pend_count[2];         // lengths of the two pending lists (by epoch parity)
  int epoch;                 // number of threshold advances
  int done;
  int advance;               // the last control step moved the threshold
  int filter_count;          // length of the pending list being filtered
  int peak;                  // largest queue of the current threshold step
  double T;                  // threshold on the first level of the time
  unsigned long long minrej; // bits of the smallest candidate queued since
                             // the last advance (times are >= 0)
  unsigned long long minkeep;// bits of the smallest candidate kept waiting
  int arrived;               // blocks of the current k_fmm_apply that finished
};

struct Lists {
  int* active;               // two lists of n points (by pass parity)
  int* stamp;                // pass that last queued a point
  int* pending;              // two lists of n points (by epoch parity)
  int* pend_stamp;           // epoch + 1 that last queued a point
  double* new_d;             // per slot of the active list: the evaluated value,
  Time3* new_t;              //   time and what to apply (bit 0: evaluated,
  unsigned char* new_f;      //   bit 1: an extension field changed)
};

// grid coordinates of point o (the entry points limit grids to 2^31 - 1
// points, so 32-bit division is exact)
__device__ __forceinline__ void point_coords(long o, int nx, int ny, int c[3]) {
  const unsigned u = (unsigned)o, q = u / (unsigned)nx;
  c[0] = (int)(u - q * (unsigned)nx);
  c[1] = (int)(q % (unsigned)ny);
  c[2] = (int)(q / (unsigned)ny);
}

// the smallest of the warp's values (every lane takes part)
__device__ __forceinline__ unsigned long long warp_min(unsigned long long v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
    v = o < v ? o : v;
  }
  return v;
}

__device__ __forceinline__ void push_once(long p, int stamp_val, int* stamp, int* list,
                                          int* count) {
  if (atomicExch(stamp + p, stamp_val) != stamp_val) list[atomicAdd(count, 1)] = (int)p;
}

// The first active list: the free points next to the front.
__global__ void k_fmm_seed(const unsigned char* st, int nx, int ny, int nz, Lists L,
                           Ctrl* ctrl) {
  const long n = (long)nx * ny * nz;
  const long s[3] = {1L, (long)nx, (long)nx * ny};
  const int nn[3] = {nx, ny, nz};
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n;
       o += (long)gridDim.x * blockDim.x) {
    if (st[o] != kFree) continue;
    int c[3];
    point_coords(o, nx, ny, c);
    bool near = false;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const int dir = q >> 1, sg = (q & 1) ? 1 : -1;
      const int c1 = c[dir] + sg;
      if (c1 >= 0 && c1 < nn[dir] && st[o + sg * s[dir]] == kFront) near = true;
    }
    if (near) push_once(o, 1, L.stamp, L.active, &ctrl->count[0]);
  }
}

// The first half of a pass over the active list (count[pass & 1]): each
// point's value and time from the values before the pass, into the list's
// side arrays, with what changed; rejected points join the pending list.
// After a threshold advance it also filters the last epoch's pending list
// (below the main loop).
template <int ORDER, bool EIK>
__global__ void __launch_bounds__(128, ORDER == 1 ? 4 : 3)
k_fmm_pass(double* d, Time3* tm, const unsigned char* st, int nx, int ny, int nz,
           double i2x, double i2y, double i2z, Lists L, Ctrl* ctrl, ExtSet X, Eik E) {
  // the control words, and the first slot of both active lists (the pass
  // number picks one), are loaded together: no load waits on another
  const long n = (long)nx * ny * nz;
  const int w_first = blockIdx.x * blockDim.x + threadIdx.x;
  const int first0 = w_first < n ? L.active[w_first] : 0;
  const int first1 = w_first < n ? L.active[n + w_first] : 0;
  const int it = ctrl->pass;
  const int count0 = ctrl->count[0], count1 = ctrl->count[1];
  const int ep = ctrl->epoch;
  const double T = ctrl->T;
  const int advance = ctrl->advance, filter_count = ctrl->filter_count;
  const int par = it & 1;
  const int count = par ? count1 : count0;
  const int* cur = L.active + par * n;
  int* pend = L.pending + (ep & 1) * n;
  int* pend_count = &ctrl->pend_count[ep & 1];
  const double i2[3] = {i2x, i2y, i2z};
  const int nn[3] = {nx, ny, nz};
  const long s[3] = {1L, (long)nx, (long)nx * ny};
  unsigned long long minrej = ~0ULL;
  for (int w = w_first; w < count; w += gridDim.x * blockDim.x) {
    const long o = w == w_first ? (par ? first1 : first0) : cur[w];
    // only free points are ever queued; the status, value and time of the
    // point itself are loaded beside its stencil
    const unsigned char self = st[o];
    const double old = d[o];
    const Time3 told = tm[o];
    int c[3];
    point_coords(o, nx, ny, c);
    Stencil nb;
    double val;
    Time3 tv, trig;
    long itrig;
    int incl;
    bool trig_free;
    bool ext_changed = false;
    const bool reached = fmm_point<ORDER, EIK>(d, tm, st, o, c, nn, s, i2, E, nb, val, tv,
                                               incl, trig, itrig, trig_free);
    if (self != kFree) {
      L.new_f[w] = 0;
      continue;
    }
    if (!reached) {
      // no neighbour is reached (any more): no update, the point is unreached
      val = copysign(INFINITY, old);
      tv = Time3{INFINITY, INFINITY, INFINITY};
    } else if (!(tv.a <= T)) {
      // accepted after the threshold: a candidate only, waiting for T
      val = copysign(INFINITY, old);
      push_once(o, ep + 1, L.pend_stamp, pend, pend_count);
      const unsigned long long bits = __double_as_longlong(tv.a);
      minrej = bits < minrej ? bits : minrej;
    } else if (!EIK && X.nf) {
      ext_changed = fmm_ext<ORDER>(nb, incl, trig, itrig, trig_free, val, i2, X, o, s);
    }
    // what k_fmm_apply does with the slot: bit 0 store the value and time,
    // bit 1 queue the readers (the change is visible: the value is finite
    // before or after, or an extension field changed)
    unsigned char f = 0;
    if (ext_changed || !(val == old && tequal(tv, told))) {
      f = 1;
      if (ext_changed || fabs(old) <= DBL_MAX || fabs(val) <= DBL_MAX) f |= 2;
    }
    L.new_d[w] = val;
    L.new_t[w] = tv;
    L.new_f[w] = f;
  }
  minrej = warp_min(minrej);
  if ((threadIdx.x & 31) == 0 && minrej != ~0ULL) atomicMin(&ctrl->minrej, minrej);
  // After a threshold advance (the control step that ended the last pass):
  // the pending points of the last epoch that the new threshold reaches join
  // the queue of the next pass beside the readers k_fmm_apply queues (same
  // list, same stamp); the others wait in this epoch's pending list.  Values
  // and times do not change during this kernel, so the test reads them as
  // the pass does.
  if (advance) {
    const int* src = L.pending + ((ep - 1) & 1) * n;
    int* next = L.active + (par ^ 1) * n;
    unsigned long long mk = ~0ULL;
    for (int w = w_first; w < filter_count; w += gridDim.x * blockDim.x) {
      const long o = src[w];
      if (fabs(d[o]) <= DBL_MAX) continue;   // reached since
      const double t = tm[o].a;
      if (t <= T) {
        push_once(o, it + 2, L.stamp, next, &ctrl->count[par ^ 1]);
      } else if (t < INFINITY) {
        push_once(o, ep + 1, L.pend_stamp, pend, pend_count);
        const unsigned long long bits = __double_as_longlong(t);
        mk = bits < mk ? bits : mk;
      }
    }
    mk = warp_min(mk);
    if ((threadIdx.x & 31) == 0 && mk != ~0ULL) atomicMin(&ctrl->minkeep, mk);
  }
}

// Between passes (the last block of k_fmm_apply, one thread).  Each
// threshold step has a burst of large passes and then a long tail of small
// ones as the last revisions settle; the threshold need not wait for that
// tail (the fixed point does not depend on when T moves, only the amount of
// revision does).  So once the queued points fall to 1/kTailFraction of the
// step's largest pass, the threshold moves to max(T + delta, smallest
// waiting candidate) and the pending list is filtered (by the next pass
// kernel) into the queue after it.  With nothing queued and nothing waiting, the solve is
// done.  The words are read volatile: other blocks of the same launch wrote
// the queue length.
constexpr int kTailFraction = 8;

__device__ void fmm_control(double delta, volatile Ctrl* ctrl) {
  // every word in one round of loads (none waits on another)
  const int done = ctrl->done, pass = ctrl->pass, peak0 = ctrl->peak, ep = ctrl->epoch;
  const int count0 = ctrl->count[0], count1 = ctrl->count[1];
  const int pend0 = ctrl->pend_count[0], pend1 = ctrl->pend_count[1];
  const unsigned long long rej = ctrl->minrej, keep = ctrl->minkeep;
  const double T = ctrl->T;
  if (done) return;
  const int par = pass & 1;
  const int queued = par ? count0 : count1;
  const int peak = queued > peak0 ? queued : peak0;
  int advance = 0;
  if ((long)queued * kTailFraction <= peak) {
    const int np = (ep & 1) ? pend1 : pend0;
    if (np == 0) {
      if (queued == 0) ctrl->done = 1;
    } else {
      const unsigned long long m = rej < keep ? rej : keep;
      const double lo = __longlong_as_double((long long)m);
      const double step = T + delta;
      ctrl->T = lo > step ? lo : step;
      advance = 1;
      ctrl->filter_count = np;
      ctrl->pend_count[(ep & 1) ^ 1] = 0;
      ctrl->epoch = ep + 1;
      ctrl->minrej = __double_as_longlong(INFINITY);
      ctrl->minkeep = __double_as_longlong(INFINITY);
    }
  }
  ctrl->peak = advance ? queued : peak;
  ctrl->advance = advance;
  ctrl->count[par] = 0;
  ctrl->pass = pass + 1;
}

// The second half of a pass: the values and times evaluated by k_fmm_pass are
// stored, and the points whose stencil reads a changed point are queued.
// Evaluating every point of a pass from the values before it (rather than
// in place, while others change) keeps the passes from cycling: read in
// place, a half-written neighbour can sustain an oscillation that sequential
// or synchronous sweeps never enter.
//
// The kernel is a short chain of memory round trips, so it is laid out to
// keep each round in flight at once: a warp takes 32 consecutive slots; the
// slot words load together; the readers' statuses load together; their
// stamps are exchanged together; and the warp reserves its queue entries
// with one atomic.  The block that finishes last runs the threshold control.
template <int ORDER>
__global__ void __launch_bounds__(256)
k_fmm_apply(double* d, Time3* tm, const unsigned char* st, int nx, int ny, int nz, Lists L,
            Ctrl* ctrl, double delta) {
  constexpr int kReaders = 6 * ORDER;
  const long n = (long)nx * ny * nz;
  const int lane = threadIdx.x & 31;
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  // the words of the first slot (both active lists for the point: the pass
  // number picks one) load beside the control words
  const int w_first = warp * 32 + lane;
  unsigned char f_first = 0;
  int first0 = 0, first1 = 0;
  double d_first = 0;
  Time3 t_first{0, 0, 0};
  if (w_first < n) {
    f_first = L.new_f[w_first];
    first0 = L.active[w_first];
    first1 = L.active[n + w_first];
    d_first = L.new_d[w_first];
    t_first = L.new_t[w_first];
  }
  const int it = ctrl->pass;
  const int count0 = ctrl->count[0], count1 = ctrl->count[1];
  const int par = it & 1;
  const int count = par ? count1 : count0;
  const int* cur = L.active + par * n;
  int* next = L.active + (par ^ 1) * n;
  int* next_count = &ctrl->count[par ^ 1];
  const int nn[3] = {nx, ny, nz};
  const long s[3] = {1L, (long)nx, (long)nx * ny};
  // the loop bound is the same for the 32 lanes of a warp
  for (int w0 = warp * 32; w0 < count; w0 += nwarps * 32) {
    const int w = w0 + lane;
    unsigned char f = 0;
    long o = 0;
    double val = 0;
    Time3 tv{0, 0, 0};
    if (w < count) {
      if (w == w_first) {
        f = f_first;
        o = par ? first1 : first0;
        val = d_first;
        tv = t_first;
      } else {
        f = L.new_f[w];
        o = cur[w];
        val = L.new_d[w];
        tv = L.new_t[w];
      }
    }
    if (f & 1) {
      d[o] = val;
      tm[o] = tv;
    }
    // the free points whose stencil reads this one
    long on[kReaders];
    unsigned won = 0;
    if (f & 2) {
      int c[3];
    point_coords(o, nx, ny, c);
      unsigned char sn[kReaders];
      unsigned cand = 0;
#pragma unroll
      for (int q = 0; q < 6; q++) {
        const int dir = q >> 1, sg = (q & 1) ? 1 : -1;
#pragma unroll
        for (int r = 1; r <= ORDER; r++) {
          const int k = q * ORDER + r - 1;
          const int cr = c[dir] + r * sg;
          const bool in = cr >= 0 && cr < nn[dir];
          on[k] = in ? o + r * sg * s[dir] : o;
          sn[k] = st[on[k]];
          if (in) cand |= 1u << k;
        }
      }
      int old[kReaders];
#pragma unroll
      for (int k = 0; k < kReaders; k++)
        if ((cand >> k & 1) && sn[k] == kFree) {
          old[k] = atomicExch(L.stamp + on[k], it + 2);
          if (old[k] != it + 2) won |= 1u << k;
        }
    }
    // one reservation for the warp's new queue entries
    const int mine = __popc(won);
    int upto = mine;
#pragma unroll
    for (int sh = 1; sh < 32; sh <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, upto, sh);
      if (lane >= sh) upto += v;
    }
    const int total = __shfl_sync(0xffffffffu, upto, 31);
    if (total) {
      int base = 0;
      if (lane == 31) base = atomicAdd(next_count, total);
      base = __shfl_sync(0xffffffffu, base, 31);
      int pos = base + upto - mine;
#pragma unroll
      for (int k = 0; k < kReaders; k++)
        if (won >> k & 1) next[pos++] = (int)on[k];
    }
  }
  // the last block to finish runs the control step
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0)
    last = atomicAdd(&ctrl->arrived, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    fmm_control(delta, ctrl);
    ctrl->arrived = 0;
  }
}

// free points no front reached: the reference's default value -1 (distance
// and extension fields), or the Eikonal solver's input
__global__ void k_fmm_unreached(double* d, const unsigned char* st, long n, ExtSet X,
                                const double* phi0) {
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n;
       o += (long)gridDim.x * blockDim.x)
    if (st[o] == kFree && !(fabs(d[o]) <= DBL_MAX)) {
      d[o] = phi0 ? phi0[o] : -1.0;
      for (int f = 0; f < X.nf; f++) X.ext[f][o] = -1.0;
    }
}

// One solve on device arrays: the distance function and up to kMaxFields
// extension fields (X.nf may be 0), or with E.speed the Eikonal solution
// for the boundary data E.phi0 (dp unused).
bool solve_device(double* dd, const double* dp, const double* dm, const ExtSet& X,
                  const Eik& E, int order, const int* grid_dims, const double* dx,
                  int* passes_out, const char* R, cudaStream_t st) {
  const int nx = grid_dims[0], ny = grid_dims[1], nz = grid_dims[2];
  const long n = (long)nx * ny * nz;
  const double hmin = fmin(dx[0], fmin(dx[1], dx[2]));
  const double delta = kDeltaCells * hmin;
  // a bound on the passes for inputs without a fixed point (NaN): the
  // threshold crosses the grid in at most (diagonal / delta) steps of a
  // few passes each
  const long max_passes = 4096 + 32L * (nx + ny + nz);
  unsigned char* status = nullptr;
  Time3* tm = nullptr;
  Lists L{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  Ctrl* ctrl = nullptr;
  const size_t un = (size_t)n;
  bool ok = cuda_ok(pool_alloc((void**)&status, un, st), R) &&
            cuda_ok(pool_alloc((void**)&tm, un * sizeof(Time3), st), R) &&
            cuda_ok(pool_alloc((void**)&L.active, 2 * un * sizeof(int), st), R) &&
            cuda_ok(pool_alloc((void**)&L.pending, 2 * un * sizeof(int), st), R) &&
            cuda_ok(pool_alloc((void**)&L.stamp, un * sizeof(int), st), R) &&
            cuda_ok(pool_alloc((void**)&L.pend_stamp, un * sizeof(int), st), R) &&
            cuda_ok(pool_alloc((void**)&L.new_d, un * sizeof(double), st), R) &&
            cuda_ok(pool_alloc((void**)&L.new_t, un * sizeof(Time3), st), R) &&
            cuda_ok(pool_alloc((void**)&L.new_f, un, st), R) &&
            cuda_ok(pool_alloc((void**)&ctrl, sizeof(Ctrl), st), R);
  Ctrl h_ctrl{};
  h_ctrl.T = delta;
  h_ctrl.minrej = 0x7ff0000000000000ULL;   // +infinity
  h_ctrl.minkeep = 0x7ff0000000000000ULL;
  int sms = 148;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int elem_blocks = (int)((n + 255) / 256 < 8 * sms ? (n + 255) / 256 : 8 * sms);
  if (ok) {
    ok = cuda_ok(cudaMemsetAsync(L.stamp, 0, un * sizeof(int), st), R) &&
         cuda_ok(cudaMemsetAsync(L.pend_stamp, 0, un * sizeof(int), st), R) &&
         cuda_ok(cudaMemcpyAsync(ctrl, &h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, st), R);
  }
  if (ok) {
    const dim3 blk(32, 4, 1);
    const dim3 grid3((nx + 31) / 32, (ny + 3) / 4, nz < 65535 ? nz : 65535);
    if (E.speed)
      k_eik_front<<<elem_blocks, 256, 0, st>>>(dd, tm, status, E.phi0, E.speed, dm, n);
    else
      k_fmm_front<<<grid3, blk, 0, st>>>(dd, tm, status, dp, dm, nx, ny, nz, dx[0], dx[1],
                                         dx[2], X);
    k_fmm_seed<<<elem_blocks, 256, 0, st>>>(status, nx, ny, nz, L, ctrl);
    launch_counter() += 2;
    ok = cuda_ok(cudaGetLastError(), R);
  }
  // 1/dx, squared (:1077-1078)
  double i2[3];
  for (int q = 0; q < 3; q++) {
    i2[q] = 1 / dx[q];
    i2[q] *= i2[q];
  }
  // a pass touches only the band, so a few blocks per SM cover it; the
  // grid-stride loops take any count
  const int pass_blocks = 4 * sms, apply_blocks = 2 * sms;
  const int batch = 32;
  auto launch_batch = [&](cudaStream_t s) {
    for (int q = 0; q < batch; q++) {
      if (order == 1 && !E.speed)
        k_fmm_pass<1, false><<<pass_blocks, 128, 0, s>>>(dd, tm, status, nx, ny, nz, i2[0],
                                                         i2[1], i2[2], L, ctrl, X, E);
      else if (!E.speed)
        k_fmm_pass<2, false><<<pass_blocks, 128, 0, s>>>(dd, tm, status, nx, ny, nz, i2[0],
                                                         i2[1], i2[2], L, ctrl, X, E);
      else if (order == 1)
        k_fmm_pass<1, true><<<pass_blocks, 128, 0, s>>>(dd, tm, status, nx, ny, nz, i2[0],
                                                        i2[1], i2[2], L, ctrl, X, E);
      else
        k_fmm_pass<2, true><<<pass_blocks, 128, 0, s>>>(dd, tm, status, nx, ny, nz, i2[0],
                                                        i2[1], i2[2], L, ctrl, X, E);
      if (order == 1)
        k_fmm_apply<1><<<apply_blocks, 256, 0, s>>>(dd, tm, status, nx, ny, nz, L, ctrl,
                                                     delta);
      else
        k_fmm_apply<2><<<apply_blocks, 256, 0, s>>>(dd, tm, status, nx, ny, nz, L, ctrl,
                                                     delta);
    }
  };
  // The kernels read the pass number and lists from ``ctrl``, so every batch
  // is the same sequence of launches: capture it once as a CUDA graph and
  // replay it (direct launches if the graph cannot be built).
  cudaGraphExec_t gexec = nullptr;
  if (ok) {
    cudaStream_t cs = nullptr;
    cudaGraph_t graph = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess) {
      if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        launch_batch(cs);
        if (cudaStreamEndCapture(cs, &graph) == cudaSuccess && graph) {
          if (cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess) gexec = nullptr;
          cudaGraphDestroy(graph);
        }
      }
      cudaStreamDestroy(cs);
    }
    cudaGetLastError();   // a failed capture leaves nothing behind but the error
  }
  long launched = 0;
  while (ok) {
    if (gexec) ok = cuda_ok(cudaGraphLaunch(gexec, st), R);
    else launch_batch(st);
    launched += batch;
    launch_counter() += 2 * batch;
    ok = ok && cuda_ok(cudaGetLastError(), R) &&
         cuda_ok(cudaMemcpyAsync(&h_ctrl, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st), R) &&
         cuda_ok(cudaStreamSynchronize(st), R);
    if (!ok || h_ctrl.done) break;
    if (launched >= max_passes) {
      set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": no convergence (NaN in phi?)");
      ok = false;
    }
  }
  if (ok) {
    k_fmm_unreached<<<elem_blocks, 256, 0, st>>>(dd, status, n, X, E.phi0);
    ++launch_counter();
    ok = cuda_ok(cudaGetLastError(), R);
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  for (void* q : {(void*)status, (void*)tm, (void*)L.active, (void*)L.pending,
                  (void*)L.stamp, (void*)L.pend_stamp, (void*)L.new_d, (void*)L.new_t,
                  (void*)L.new_f, (void*)ctrl})
    if (q) cudaFreeAsync(q, st);
  if (passes_out) *passes_out = h_ctrl.pass;
  return ok;
}

// computeExtensionFields3d / computeDistanceFunction3d on host or device
// arrays: argument checks, staging, and one solve per group of kMaxFields
// fields (each solve recomputes the same distance function).
int extension3d(double* distance, double** ext, const double* phi, const double* mask,
                double* const* src, const double* emask, int nf, int order,
                const int* grid_dims, const double* dx, int* passes_out, const char* R) {
  clear_error();
  if (!distance || !phi || !grid_dims || !dx || (nf > 0 && (!ext || !src))) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  for (int k = 0; k < nf; k++)
    if (!ext[k] || !src[k]) {
      set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null field pointer");
      return LSMGPU_ERR_NULL_POINTER;
    }
  if (nf < 0) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": negative field count");
    return LSMGPU_ERR_INVALID_VALUE;
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
  if (!(dx[0] > 0) || !(dx[1] > 0) || !(dx[2] > 0) || !(dx[0] < INFINITY) ||
      !(dx[1] < INFINITY) || !(dx[2] < INFINITY)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": dx must be positive and finite");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  if ((long)nx * ny * nz > 0x7fffffffL) {
    set_error(LSMGPU_ERR_INVALID_BOX, std::string(R) + ": more than 2^31 - 1 points");
    return LSMGPU_ERR_INVALID_BOX;
  }
  cudaStream_t st = cur_stream();
  Staging stg(st);
  const Box b{{0, 0, 0}, {nx, ny, nz}};
  double* dd = (double*)stg.add(distance, b, 8, kOutFull, "distance_function", R);
  const double* dp = dd ? (const double*)stg.add(phi, b, 8, kIn, "phi", R) : nullptr;
  const double* dm = nullptr;
  if (dp && mask) dm = (const double*)stg.add(mask, b, 8, kIn, "mask", R);
  const double* dem = nullptr;
  if (dp && emask) dem = (const double*)stg.add(emask, b, 8, kIn, "extension_mask", R);
  if (!dd || !dp || (mask && !dm) || (emask && !dem)) return lsmgpu_peek_last_error();
  int group = 0;
  do {
    ExtSet X{};
    X.emask = dem;
    X.nf = nf - group < kMaxFields ? nf - group : kMaxFields;
    for (int k = 0; k < X.nf; k++) {
      X.ext[k] = (double*)stg.add(ext[group + k], b, 8, kOutFull, "extension_field", R);
      X.src[k] = X.ext[k] ? (const double*)stg.add(src[group + k], b, 8, kIn, "source_field",
                                                   R)
                          : nullptr;
      if (!X.ext[k] || !X.src[k]) return lsmgpu_peek_last_error();
    }
    if (!solve_device(dd, dp, dm, X, Eik{nullptr, nullptr}, order, grid_dims, dx, passes_out,
                      R, st))
      return lsmgpu_peek_last_error() ? lsmgpu_peek_last_error() : LSMGPU_ERR_CUDA;
    group += X.nf;
  } while (group < nf);
  return stg.finish(R) ? LSMGPU_SUCCESS : LSMGPU_ERR_CUDA;
}

// solveEikonalEquation3d on host or device arrays: phi holds the boundary
// data on input and the solution on output.
int eikonal3d(double* phi, const double* speed, const double* mask, int order,
              const int* grid_dims, const double* dx, int* passes_out, const char* R) {
  clear_error();
  if (!phi || !speed || !grid_dims || !dx) {
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
  if (!(dx[0] > 0) || !(dx[1] > 0) || !(dx[2] > 0) || !(dx[0] < INFINITY) ||
      !(dx[1] < INFINITY) || !(dx[2] < INFINITY)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": dx must be positive and finite");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  const long n = (long)nx * ny * nz;
  if (n > 0x7fffffffL) {
    set_error(LSMGPU_ERR_INVALID_BOX, std::string(R) + ": more than 2^31 - 1 points");
    return LSMGPU_ERR_INVALID_BOX;
  }
  cudaStream_t st = cur_stream();
  Staging stg(st);
  const Box b{{0, 0, 0}, {nx, ny, nz}};
  double* dd = (double*)stg.add(phi, b, 8, kInOut, "phi", R);
  const double* df = dd ? (const double*)stg.add(speed, b, 8, kIn, "speed", R) : nullptr;
  const double* dm = nullptr;
  if (df && mask) dm = (const double*)stg.add(mask, b, 8, kIn, "mask", R);
  if (!dd || !df || (mask && !dm)) return lsmgpu_peek_last_error();
  double* phi0 = nullptr;
  bool ok = cuda_ok(pool_alloc((void**)&phi0, (size_t)n * sizeof(double), st), R) &&
            cuda_ok(cudaMemcpyAsync(phi0, dd, (size_t)n * sizeof(double),
                                    cudaMemcpyDeviceToDevice, st), R);
  ok = ok && solve_device(dd, nullptr, dm, ExtSet{}, Eik{df, phi0}, order, grid_dims, dx,
                          passes_out, R, st);
  if (phi0) cudaFreeAsync(phi0, st);
  if (!ok) return lsmgpu_peek_last_error() ? lsmgpu_peek_last_error() : LSMGPU_ERR_CUDA;
  return stg.finish(R) ? LSMGPU_SUCCESS : LSMGPU_ERR_CUDA;
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
  const int rc = extension3d(distance_function, nullptr, phi, mask, nullptr, nullptr, 0,
                             spatial_discretization_order, grid_dims, dx, nullptr,
                             "computeDistanceFunction3d");
  return rc == LSMGPU_SUCCESS ? 0 : -1;
}

// lsm_fast_marching_method.h:331-341, the same return codes
int computeExtensionFields3d(double* distance_function, double** extension_fields,
                             double* phi, double* mask, double** source_fields,
                             double* extension_mask, int num_extension_fields,
                             int spatial_discretization_order, int* grid_dims, double* dx) {
  if (spatial_discretization_order != 1 && spatial_discretization_order != 2) return 2;
  const int rc = extension3d(distance_function, extension_fields, phi, mask, source_fields,
                             extension_mask, num_extension_fields,
                             spatial_discretization_order, grid_dims, dx, nullptr,
                             "computeExtensionFields3d");
  return rc == LSMGPU_SUCCESS ? 0 : -1;
}

int lsmgpu_distance_function3d(double* distance_function, const double* phi,
                               const double* mask, int order, const int* grid_dims,
                               const double* dx, int* passes) {
  return extension3d(distance_function, nullptr, phi, mask, nullptr, nullptr, 0, order,
                     grid_dims, dx, passes, "lsmgpu_distance_function3d");
}

int lsmgpu_extension_fields3d(double* distance_function, double** extension_fields,
                              const double* phi, const double* mask,
                              double* const* source_fields, const double* extension_mask,
                              int num_extension_fields, int order, const int* grid_dims,
                              const double* dx, int* passes) {
  return extension3d(distance_function, extension_fields, phi, mask, source_fields,
                     extension_mask, num_extension_fields, order, grid_dims, dx, passes,
                     "lsmgpu_extension_fields3d");
}

// lsm_fast_marching_method.h:463-469, the same return codes
int solveEikonalEquation3d(double* phi, double* speed, double* mask,
                           int spatial_discretization_order, int* grid_dims, double* dx) {
  if (spatial_discretization_order != 1 && spatial_discretization_order != 2) return 2;
  const int rc = eikonal3d(phi, speed, mask, spatial_discretization_order, grid_dims, dx,
                           nullptr, "solveEikonalEquation3d");
  return rc == LSMGPU_SUCCESS ? 0 : -1;
}

int lsmgpu_eikonal3d(double* phi, const double* speed, const double* mask, int order,
                     const int* grid_dims, const double* dx, int* passes) {
  return eikonal3d(phi, speed, mask, order, grid_dims, dx, passes, "lsmgpu_eikonal3d");
}

// The 2D forms (lsm_fast_marching_method.h:124-134, 179-185, 256-262): the
// 3D solve on a grid one plane thick, on which the reference's own 2D and 3D
// routines agree bit for bit.  grid_dims and dx hold x and y; the z spacing
// is taken as dx[0] (a single plane has no z neighbours, and the threshold
// step then still follows the smallest of dx and dy).  Null arguments pass
// through as null, so the 3D checks report them.
static void plane_grid(const int* grid_dims, const double* dx, int d3[3], double h3[3],
                       const int** pd, const double** ph) {
  *pd = nullptr;
  *ph = nullptr;
  if (grid_dims) {
    d3[0] = grid_dims[0];
    d3[1] = grid_dims[1];
    d3[2] = 1;
    *pd = d3;
  }
  if (dx) {
    h3[0] = dx[0];
    h3[1] = dx[1];
    h3[2] = dx[0];
    *ph = h3;
  }
}

int computeExtensionFields2d(double* distance_function, double** extension_fields,
                             double* phi, double* mask, double** source_fields,
                             double* extension_mask, int num_extension_fields,
                             int spatial_discretization_order, int* grid_dims, double* dx) {
  if (spatial_discretization_order != 1 && spatial_discretization_order != 2) return 2;
  int d3[3];
  double h3[3];
  const int* pd;
  const double* ph;
  plane_grid(grid_dims, dx, d3, h3, &pd, &ph);
  const int rc = extension3d(distance_function, extension_fields, phi, mask, source_fields,
                             extension_mask, num_extension_fields,
                             spatial_discretization_order, pd, ph, nullptr,
                             "computeExtensionFields2d");
  return rc == LSMGPU_SUCCESS ? 0 : -1;
}

int computeDistanceFunction2d(double* distance_function, double* phi, double* mask,
                              int spatial_discretization_order, int* grid_dims,
                              double* dx) {
  if (spatial_discretization_order != 1 && spatial_discretization_order != 2) return 2;
  int d3[3];
  double h3[3];
  const int* pd;
  const double* ph;
  plane_grid(grid_dims, dx, d3, h3, &pd, &ph);
  const int rc = extension3d(distance_function, nullptr, phi, mask, nullptr, nullptr, 0,
                             spatial_discretization_order, pd, ph, nullptr,
                             "computeDistanceFunction2d");
  return rc == LSMGPU_SUCCESS ? 0 : -1;
}

int solveEikonalEquation2d(double* phi, double* speed, double* mask,
                           int spatial_discretization_order, int* grid_dims, double* dx) {
  if (spatial_discretization_order != 1 && spatial_discretization_order != 2) return 2;
  int d3[3];
  double h3[3];
  const int* pd;
  const double* ph;
  plane_grid(grid_dims, dx, d3, h3, &pd, &ph);
  const int rc = eikonal3d(phi, speed, mask, spatial_discretization_order, pd, ph, nullptr,
                           "solveEikonalEquation2d");
  return rc == LSMGPU_SUCCESS ? 0 : -1;
}

}  // extern "C"
