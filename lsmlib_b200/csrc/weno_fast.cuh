// weno_fast.cuh -- HJ-WENO5 restructured for the FP64/FP32 ALU of sm_100a.
//
// Same reconstruction as the reference (lsm_spatial_derivatives3d.f.in:
// 1292-1323) with three changes that alter only rounding:
//  * FMA contraction (the translation unit is built with --fmad=true);
//  * the nonlinear weights are normalised with a single reciprocal:
//      a_k = d_k / q_k^2,  q_k = S_k + eps
//      w_k = d_k * prod_{j!=k} q_j^2 / sum_m (d_m * prod_{j!=m} q_j^2)
//    after scaling every q_k by the power of two s = 2^-floor(log2 eps), so
//    that 1 <= q_k*s < 2^27 and the fourth-degree products stay far inside
//    the FP32 and FP64 ranges (S_k <= 33.4 max v^2 and eps >= 1e-6 max v^2);
//  * the reciprocal is the hardware seed (rcp.approx.ftz) refined: in FP64
//    by one third-order step r <- r + r (e + e^2), e = 1 - d r (the series
//    1/d = r / (1 - e) = r (1 + e + e^2 + ...) cut after e^2; the seed's
//    relative error is below 1e-6 on sm_100, so the cut term e^3 is below
//    1e-18), in FP32 by one Newton-Raphson step r <- r + r (1 - d r)
//    (Markstein, IBM J. Res. Dev. 34(1), 1990).
// The parity tests bound the difference to the reference at 1e-12 relative
// (FP64).
#pragma once
#include "common.cuh"

namespace lsmgpu {

__device__ __forceinline__ double rcp_nr(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  const double e = fma(-d, r, 1.0);
  return fma(r, fma(e, e, e), r);
}
__device__ __forceinline__ float rcp_nr(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  const float e = fmaf(-d, r, 1.0f);
  return fmaf(r, e, r);
}

// 1/sqrt(x) for x > 0: the hardware seed r (rsqrt.approx.ftz) refined.  In
// FP64 with e = 1 - x r^2, 1/sqrt(x) = r (1 - e)^(-1/2) = r (1 + e/2 +
// 3e^2/8 + 5e^3/16 + ...), cut after e^2 (the seed's relative error is below
// 1e-6 on sm_100, so the cut term is below 1e-18); in FP32 by one
// Newton-Raphson step for f(r) = 1/r^2 - x, r <- r + r (1 - x r^2) / 2
// (Markstein, IBM J. Res. Dev. 34(1), 1990).  Fast-mode arithmetic only.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double r;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  const double e = fma(-(x * r), r, 1.0);
  return fma(r * e, fma(0.375, e, 0.5), r);
}
__device__ __forceinline__ float rsqrt_nr(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  const float e = fmaf(-(x * r), r, 1.0f);
  return fmaf(0.5f * r, e, r);
}
// sqrt(x) for x >= 0 as x / sqrt(x) with rsqrt_nr; x below the normal range
// (where the ftz seed would be infinite) takes the correctly rounded sqrt
template <typename T>
__device__ __forceinline__ T sqrt_nr(T x) {
  return x >= T(sizeof(T) == 8 ? 1e-300 : 1e-30) ? x * rsqrt_nr(x) : T(sqrt(x));
}

// a * b + c with one rounding, written out where an expression has two
// products, so that every instantiation fuses the same one (the contraction
// the compiler picks can differ between inlining contexts)
__device__ __forceinline__ double fmaT(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }

// max and min for the eps maxima and the kink tests: a plain comparison in
// FP64 (CUDA's IEEE fmax of doubles, which also sorts out NaN operands, cost
// a third of the stage kernels' integer instructions; these values are
// never NaN for finite phi), the native instruction in FP32
__device__ __forceinline__ double vmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double vmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float vmin(float a, float b) { return fminf(a, b); }

// 2^-(unbiased exponent of x) for a positive normal x
__device__ __forceinline__ double inv_pow2_of(double x) {
  const int e = (__double2hiint(x) >> 20) & 0x7ff;
  return __hiloint2double((2046 - e) << 20, 0);
}
__device__ __forceinline__ float inv_pow2_of(float x) {
  const int e = (__float_as_int(x) >> 23) & 0xff;
  return __int_as_float((254 - e) << 23);
}

// One side of HJ-WENO5 from the five undivided differences D1..D5 in the
// reference's ordering (v_k = D_k / dx); returns the reconstruction of the
// scaled differences.  The same rearrangements as weno5_face below (rounding
// only): the weights see only ratios of D (scaling by 1/dx is applied once
// at the end), eps is taken from max|D|, the S_k and eps are taken four
// times over, and with w2 = 1 - w1 - w3 and numerator and weight sum halved
//   phi = p2 + (P23 (ta - tb) + 3/2 P12 (tb - tc)) / (3 P23 + 18 P13 + 9 P12),
// P_xy = (q_x q_y)^2, ta, tb, tc the second differences of the smoothness
// indicators.
template <typename T>
__device__ __forceinline__ T weno5_side_fast(T D1, T D2, T D3, T D4, T D5, T inv) {
  const T amax = vmax(vmax(vmax(fabs(D1), fabs(D2)), vmax(fabs(D3), fabs(D4))), fabs(D5));
  const T eps = fmaT(T(4e-6), amax * amax, T(4) * Consts<T>::tiny);
  const T c13_3 = T(13.0 / 3.0);
  const T ta = fmaT(T(-2), D2, D1) + D3, tb = fmaT(T(-2), D3, D2) + D4,
          tc = fmaT(T(-2), D4, D3) + D5;
  T t = fmaT(T(3), D3, fmaT(T(-4), D2, D1));
  const T S1 = fmaT(c13_3 * ta, ta, t * t);
  t = D2 - D4;
  const T S2 = fmaT(c13_3 * tb, tb, t * t);
  t = fmaT(T(-4), D4, T(3) * D3) + D5;
  const T S3 = fmaT(c13_3 * tc, tc, t * t);
  const T sc = inv_pow2_of(eps);
  const T es = eps * sc;
  const T q1 = fmaT(S1, sc, es), q2 = fmaT(S2, sc, es), q3 = fmaT(S3, sc, es);
  const T Q1 = q1 * q1, Q2 = q2 * q2, Q3 = q3 * q3;
  const T P23 = Q2 * Q3, P13 = Q1 * Q3, P12 = Q1 * Q2;
  const T num = fmaT(T(1.5), P12 * (tb - tc), P23 * (ta - tb));
  const T den = fmaT(T(3), P23, fmaT(T(18), P13, T(9) * P12));
  const T p2 = fmaT(T(1.0 / 3.0), D4, fmaT(T(-1.0 / 6.0), D2, T(5.0 / 6.0) * D3));
  return fmaT(num, rcp_nr(den), p2) * inv;
}

// Weights and combination of one side from its smoothness indicators,
// candidates and eps (see the header comment for the scaled single-reciprocal
// normalisation).
template <typename T>
__device__ __forceinline__ T weno5_weigh(T S1, T S2, T S3, T p1, T p2, T p3,
                                         T eps) {
  const T sc = inv_pow2_of(eps);
  const T es = eps * sc;
  const T q1 = S1 * sc + es, q2 = S2 * sc + es, q3 = S3 * sc + es;
  const T Q1 = q1 * q1, Q2 = q2 * q2, Q3 = q3 * q3;
  const T n1 = T(0.1) * (Q2 * Q3), n2 = T(0.6) * (Q1 * Q3), n3 = T(0.3) * (Q1 * Q2);
  const T r = rcp_nr(n1 + n2 + n3);
  return (n1 * p1 + n2 * p2 + n3 * p3) * r;
}

// Plus and minus HJ-WENO5 derivatives of one axis from seven consecutive
// values w[0..6] = phi(c-3..c+3), computed together: the six scaled
// differences V_m = (w[m+1]-w[m])/dx, their squares, the common part of the
// two eps maxima and two of the three curvature terms (a-2b+c)^2 of each
// side are shared.  minus uses v1..v5 = V0..V4, plus uses v1..v5 = V5..V1
// (lsm_spatial_derivatives3d.f.in:1286-1290, :1330-1334).  When KINK64 is
// set (FP32 form), a side whose smoothness indicators differ by more than a
// factor 1e3 is recomputed in FP64 from the phi values.
template <typename T, bool KINK64>
__device__ __forceinline__ void weno5_pm_fast(const T* w, T inv, T& vp, T& vm) {
  T V[6], s[6];
#pragma unroll
  for (int m = 0; m < 6; m++) {
    V[m] = (w[m + 1] - w[m]) * inv;
    s[m] = V[m] * V[m];
  }
  const T mid = vmax(vmax(s[1], s[2]), vmax(s[3], s[4]));
  const T eps_m = T(1e-6) * vmax(mid, s[0]) + Consts<T>::tiny;
  const T eps_p = T(1e-6) * vmax(mid, s[5]) + Consts<T>::tiny;
  const T c13_12 = T(13.0 / 12.0), c14 = T(0.25);
  T t;
  t = V[0] - T(2) * V[1] + V[2]; const T cA = t * t;
  t = V[1] - T(2) * V[2] + V[3]; const T cB = t * t;
  t = V[2] - T(2) * V[3] + V[4]; const T cC = t * t;
  t = V[3] - T(2) * V[4] + V[5]; const T cD = t * t;
  // minus side
  t = V[0] - T(4) * V[1] + T(3) * V[2];
  const T mS1 = c13_12 * cA + c14 * (t * t);
  t = V[1] - V[3];
  const T mS2 = c13_12 * cB + c14 * (t * t);
  t = T(3) * V[2] - T(4) * V[3] + V[4];
  const T mS3 = c13_12 * cC + c14 * (t * t);
  // plus side
  t = V[5] - T(4) * V[4] + T(3) * V[3];
  const T pS1 = c13_12 * cD + c14 * (t * t);
  t = V[4] - V[2];
  const T pS2 = c13_12 * cC + c14 * (t * t);
  t = T(3) * V[3] - T(4) * V[2] + V[1];
  const T pS3 = c13_12 * cB + c14 * (t * t);
  const T a = T(1.0 / 3.0), b = T(7.0 / 6.0), c = T(11.0 / 6.0), d = T(1.0 / 6.0),
          e = T(5.0 / 6.0);
  const T mp1 = a * V[0] - b * V[1] + c * V[2];
  const T mp2 = -d * V[1] + e * V[2] + a * V[3];
  const T mp3 = a * V[2] + e * V[3] - d * V[4];
  const T pp1 = a * V[5] - b * V[4] + c * V[3];
  const T pp2 = -d * V[4] + e * V[3] + a * V[2];
  const T pp3 = a * V[3] + e * V[2] - d * V[1];
  vm = weno5_weigh(mS1, mS2, mS3, mp1, mp2, mp3, eps_m);
  vp = weno5_weigh(pS1, pS2, pS3, pp1, pp2, pp3, eps_p);
  if (KINK64) {
    const T scale = vmax(mid, vmax(s[0], s[5]));
    const bool km = vmax(vmax(mS1, mS2), mS3) > T(1e3) * vmin(vmin(mS1, mS2), mS3) + T(1e-4) * scale;
    const bool kp = vmax(vmax(pS1, pS2), pS3) > T(1e3) * vmin(vmin(pS1, pS2), pS3) + T(1e-4) * scale;
    if (km || kp) {
      double wd[7];
#pragma unroll
      for (int m = 0; m < 7; m++) wd[m] = (double)w[m];
      double dp, dm;
      weno5_pm_fast<double, false>(wd, (double)inv, dp, dm);
      if (km) vm = (T)dm;
      if (kp) vp = (T)dp;
    }
  }
}

// FP64 recomputation of one face for the FP32 form (defined below; kept out
// of line so that the rarely taken path does not grow every call site)
static __device__ __noinline__ float2 weno5_face_fp64(float u0, float u1, float u2,
                                                     float u3, float u4, float u5,
                                                     float inv);

// Per-axis constants of weno5_face: 1/dx and the weights of the middle
// candidate scaled by it.
template <typename T>
struct FaceConst {
  T inv, c3, c56, c16;   // 1/dx, 1/(3dx), 5/(6dx), 1/(6dx)
};
template <typename T>
__host__ __device__ inline FaceConst<T> face_const(T inv) {
  return {inv, inv * T(1.0 / 3.0), inv * T(5.0 / 6.0), inv * T(1.0 / 6.0)};
}

// The two HJ-WENO5 values that share the face between cells c and c+1, from
// u[0..5] = phi(c-2..c+3): vp = phi^+(c) and vm = phi^-(c+1).  Both read the
// same five differences V1..V5 (faces c-3/2..c+5/2), minus in the order
// V1..V5 and plus in the order V5..V1 (lsm_spatial_derivatives3d.f.in:
// 1286-1290, :1330-1334), so they share eps, the three smoothness indicators
// Sa, Sb, Sc (plus sees them as S3, S2, S1) and the products
// P_xy = (q_x q_y)^2 of the single-reciprocal normalisation; only the
// assignment of the linear weights {0.1, 0.6, 0.3} differs.  With
// w2 = 1 - w1 - w3 the reconstruction is
//   phi = p2 + w1 (p1 - p2) + w3 (p3 - p2),
//   p1 - p2 = (ta - tb)/3,  p3 - p2 = (tb - tc)/6,
// where ta, tb, tc are the second differences of V already formed for the
// smoothness indicators; for the reversed (plus) stencil the two third
// differences swap and change sign.  So
//   vm = p2m + (2 Pbc T1 + 3 Pab T2) / (60 sm),
//   vp = p2p - (2 Pab T2 + 3 Pbc T1) / (60 sp),
// with T1 = ta - tb, T2 = tb - tc and sm, sp the weight sums.  Three more
// rearrangements change only rounding:
//  * the reconstruction is homogeneous of degree one in V and its weights
//    of degree zero (but for the floor of eps), so it runs on the undivided
//    differences D = u[m+1] - u[m] and the two results are scaled by 1/dx
//    once;
//  * the eps maximum is max|D| squared (rounding is monotone, so this is
//    exactly the largest square);
//  * in FP64 one reciprocal of the product of the two weight sums serves
//    both sides (the products stay below 2^230; in FP32 they would overflow,
//    so FP32 takes two).
// When KINK64 is set (FP32 form) a face whose indicators differ by more than
// a factor 1e3 is recomputed in FP64.  Three further rearrangements, again
// only rounding:
//  * the S_k and eps enter the weights only through ratios of the q_k, so
//    all four are taken four times over: S_k = 13/3 t1^2 + t2^2 (the
//    reference's 13/12 t1^2 + 1/4 t2^2) and eps = 4e-6 max D^2 + 4 tiny;
//  * numerators and weight sums are halved: vm = p2m + (A + 3/2 B) / (3 Pbc +
//    18 Pac + 9 Pab), vp = p2p - (B + 3/2 A) / (3 Pab + 18 Pac + 9 Pbc), the
//    18 Pac shared;
//  * 1/dx is folded into the middle candidate's weights (FaceConst) and
//    into the one reciprocal.
// LMAX: the eps maximum grouped as max(|D1|, max(|D2|..|D5|)) instead of
// max(max(|D1|..|D4|), |D5|) -- the same value; a face evaluated with LMAX
// beside the face one cell on (without) shares the inner four-way maximum.
template <typename T, bool KINK64, bool LMAX = false>
__device__ __forceinline__ void weno5_face(const T* u, const FaceConst<T>& k, T& vp, T& vm) {
  const T V1 = u[1] - u[0], V2 = u[2] - u[1], V3 = u[3] - u[2], V4 = u[4] - u[3],
          V5 = u[5] - u[4];
  const T amax = LMAX ? vmax(fabs(V1), vmax(vmax(fabs(V2), fabs(V3)), vmax(fabs(V4), fabs(V5))))
                      : vmax(vmax(vmax(fabs(V1), fabs(V2)), vmax(fabs(V3), fabs(V4))), fabs(V5));
  const T m = amax * amax;
  // four times the reference's 1e-6 max(v^2) + tiny, in units of the
  // undivided differences (the floor, reached only where every |D| < 1e-46,
  // is kept in these units)
  const T eps = fmaT(T(4e-6), m, T(4) * Consts<T>::tiny);
  const T c13_3 = T(13.0 / 3.0);
  const T ta = fmaT(T(-2), V2, V1) + V3, tb = fmaT(T(-2), V3, V2) + V4,
          tc = fmaT(T(-2), V4, V3) + V5;
  T t = fmaT(T(3), V3, fmaT(T(-4), V2, V1));
  const T Sa = fmaT(c13_3 * ta, ta, t * t);
  t = V2 - V4;
  const T Sb = fmaT(c13_3 * tb, tb, t * t);
  t = fmaT(T(-4), V4, T(3) * V3) + V5;
  const T Sc = fmaT(c13_3 * tc, tc, t * t);
  if (KINK64) {
    const T mx = vmax(vmax(Sa, Sb), Sc), mn = vmin(vmin(Sa, Sb), Sc);
    if (mx > T(1e3) * mn + T(4e-4) * m) {
      if constexpr (sizeof(T) == 4) {
        const float2 r = weno5_face_fp64(u[0], u[1], u[2], u[3], u[4], u[5], k.inv);
        vp = r.x;
        vm = r.y;
        return;
      }
    }
  }
  const T sc = inv_pow2_of(eps);
  const T es = eps * sc;
  const T qa = fmaT(Sa, sc, es), qb = fmaT(Sb, sc, es), qc = fmaT(Sc, sc, es);
  const T Qa = qa * qa, Qb = qb * qb, Qc = qc * qc;
  const T Pbc = Qb * Qc, Pac = Qa * Qc, Pab = Qa * Qb;
  const T A = Pbc * (ta - tb), B = Pab * (tb - tc);
  const T num_m = fmaT(T(1.5), B, A), num_p = fmaT(T(1.5), A, B);
  const T e3 = k.c56 * V3;
  const T p2m = fmaT(k.c3, V4, fmaT(-k.c16, V2, e3));
  const T p2p = fmaT(k.c3, V2, fmaT(-k.c16, V4, e3));
  // 30 sm and 30 sp
  const T p18 = T(18) * Pac;
  const T sm = fmaT(T(3), Pbc, fmaT(T(9), Pab, p18));
  const T sp = fmaT(T(3), Pab, fmaT(T(9), Pbc, p18));
  if constexpr (sizeof(T) == 8) {
    const T r = rcp_nr(sm * sp) * k.inv;
    vm = fmaT(num_m, sp * r, p2m);
    vp = fmaT(-num_p, sm * r, p2p);
  } else {
    vm = fmaT(num_m, rcp_nr(sm) * k.inv, p2m);
    vp = fmaT(-num_p, rcp_nr(sp) * k.inv, p2p);
  }
}
template <typename T, bool KINK64>
__device__ __forceinline__ void weno5_face(const T* u, T inv, T& vp, T& vm) {
  weno5_face<T, KINK64>(u, face_const(inv), vp, vm);
}

// weno5_face<float> for two independent faces at once, one per lane of a
// float2 (u[m].x and u[m].y: phi(c-2+m) of each face), on the packed FP32x2
// arithmetic of sm_100 (__ffma2_rn, __fadd2_rn, __fmul2_rn: two IEEE single
// operations per instruction).  The same formulas as weno5_face with explicit
// fused multiply-adds; the eps maximum, the power-of-two scaling and the
// reciprocal seeds stay per lane.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b, rounded once (b * -1 is exact)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }

__device__ __forceinline__ void weno5_face2(const float2* u, float inv, float2& vp, float2& vm) {
  const float2 V1 = sub2(u[1], u[0]), V2 = sub2(u[2], u[1]), V3 = sub2(u[3], u[2]),
               V4 = sub2(u[4], u[3]), V5 = sub2(u[5], u[4]);
  float2 amax;
  amax.x = vmax(vmax(vmax(fabsf(V1.x), fabsf(V2.x)), vmax(fabsf(V3.x), fabsf(V4.x))), fabsf(V5.x));
  amax.y = vmax(vmax(vmax(fabsf(V1.y), fabsf(V2.y)), vmax(fabsf(V3.y), fabsf(V4.y))), fabsf(V5.y));
  const float2 m = mul2(amax, amax);
  // S_k and eps four times over, as in weno5_face
  const float2 eps = fma2(f2(4e-6f), m, f2(4.0f * Consts<float>::tiny));
  const float2 c13_3 = f2(13.0f / 3.0f);
  const float2 ta = add2(fma2(f2(-2.0f), V2, V1), V3);
  const float2 tb = add2(fma2(f2(-2.0f), V3, V2), V4);
  const float2 tc = add2(fma2(f2(-2.0f), V4, V3), V5);
  float2 t = fma2(f2(3.0f), V3, fma2(f2(-4.0f), V2, V1));
  const float2 Sa = fma2(mul2(c13_3, ta), ta, mul2(t, t));
  t = sub2(V2, V4);
  const float2 Sb = fma2(mul2(c13_3, tb), tb, mul2(t, t));
  t = add2(fma2(f2(-4.0f), V4, mul2(f2(3.0f), V3)), V5);
  const float2 Sc = fma2(mul2(c13_3, tc), tc, mul2(t, t));
  const float2 sc = make_float2(inv_pow2_of(eps.x), inv_pow2_of(eps.y));
  const float2 es = mul2(eps, sc);
  const float2 qa = fma2(Sa, sc, es), qb = fma2(Sb, sc, es), qc = fma2(Sc, sc, es);
  const float2 Qa = mul2(qa, qa), Qb = mul2(qb, qb), Qc = mul2(qc, qc);
  const float2 Pbc = mul2(Qb, Qc), Pac = mul2(Qa, Qc), Pab = mul2(Qa, Qb);
  const float2 A = mul2(Pbc, sub2(ta, tb)), B = mul2(Pab, sub2(tb, tc));
  // halved numerators and weight sums, as in weno5_face
  const float2 num_m = fma2(f2(1.5f), B, A);
  const float2 num_p = fma2(f2(1.5f), A, B);
  const float2 e3 = mul2(f2(5.0f / 6.0f), V3);
  const float2 p2m = fma2(f2(1.0f / 3.0f), V4, fma2(f2(-1.0f / 6.0f), V2, e3));
  const float2 p2p = fma2(f2(1.0f / 3.0f), V2, fma2(f2(-1.0f / 6.0f), V4, e3));
  const float2 p18 = mul2(f2(18.0f), Pac);
  const float2 sm = fma2(f2(3.0f), Pbc, fma2(f2(9.0f), Pab, p18));
  const float2 sp = fma2(f2(3.0f), Pab, fma2(f2(9.0f), Pbc, p18));
  // reciprocals: per-lane seeds, one packed Newton-Raphson step (rcp_nr)
  float2 rm, rp;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rm.x) : "f"(sm.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rm.y) : "f"(sm.y));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rp.x) : "f"(sp.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rp.y) : "f"(sp.y));
  rm = fma2(rm, fma2(mul2(f2(-1.0f), sm), rm, f2(1.0f)), rm);
  rp = fma2(rp, fma2(mul2(f2(-1.0f), sp), rp, f2(1.0f)), rp);
  vm = mul2(fma2(num_m, rm, p2m), f2(inv));
  vp = mul2(fma2(mul2(f2(-1.0f), num_p), rp, p2p), f2(inv));
}

// weno5_side_fast<float> for two independent sides at once, one per lane of
// a float2 (D[m].x and D[m].y: the five undivided differences of each side
// in its own order), with the packed FP32x2 operations of weno5_face2; the
// eps maxima, the power-of-two scalings and the reciprocal seeds stay per
// lane.
__device__ __forceinline__ float2 weno5_side2(const float2* D, float inv) {
  const float2 D1 = D[0], D2 = D[1], D3 = D[2], D4 = D[3], D5 = D[4];
  float2 amax;
  amax.x = vmax(vmax(vmax(fabsf(D1.x), fabsf(D2.x)), vmax(fabsf(D3.x), fabsf(D4.x))), fabsf(D5.x));
  amax.y = vmax(vmax(vmax(fabsf(D1.y), fabsf(D2.y)), vmax(fabsf(D3.y), fabsf(D4.y))), fabsf(D5.y));
  const float2 eps = fma2(f2(4e-6f), mul2(amax, amax), f2(4.0f * Consts<float>::tiny));
  const float2 c13_3 = f2(13.0f / 3.0f);
  const float2 ta = add2(fma2(f2(-2.0f), D2, D1), D3);
  const float2 tb = add2(fma2(f2(-2.0f), D3, D2), D4);
  const float2 tc = add2(fma2(f2(-2.0f), D4, D3), D5);
  float2 t = fma2(f2(3.0f), D3, fma2(f2(-4.0f), D2, D1));
  const float2 S1 = fma2(mul2(c13_3, ta), ta, mul2(t, t));
  t = sub2(D2, D4);
  const float2 S2 = fma2(mul2(c13_3, tb), tb, mul2(t, t));
  t = add2(fma2(f2(-4.0f), D4, mul2(f2(3.0f), D3)), D5);
  const float2 S3 = fma2(mul2(c13_3, tc), tc, mul2(t, t));
  const float2 sc = make_float2(inv_pow2_of(eps.x), inv_pow2_of(eps.y));
  const float2 es = mul2(eps, sc);
  const float2 q1 = fma2(S1, sc, es), q2 = fma2(S2, sc, es), q3 = fma2(S3, sc, es);
  const float2 Q1 = mul2(q1, q1), Q2 = mul2(q2, q2), Q3 = mul2(q3, q3);
  const float2 P23 = mul2(Q2, Q3), P13 = mul2(Q1, Q3), P12 = mul2(Q1, Q2);
  const float2 num = fma2(f2(1.5f), mul2(P12, sub2(tb, tc)), mul2(P23, sub2(ta, tb)));
  const float2 den = fma2(f2(3.0f), P23, fma2(f2(18.0f), P13, mul2(f2(9.0f), P12)));
  const float2 p2 = fma2(f2(1.0f / 3.0f), D4, fma2(f2(-1.0f / 6.0f), D2, mul2(f2(5.0f / 6.0f), D3)));
  float2 r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(den.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(den.y));
  r = fma2(r, fma2(mul2(f2(-1.0f), den), r, f2(1.0f)), r);
  return mul2(fma2(num, r, p2), f2(inv));
}

static __device__ __noinline__ float2 weno5_face_fp64(float u0, float u1, float u2,
                                                     float u3, float u4, float u5,
                                                     float inv) {
  const double ud[6] = {u0, u1, u2, u3, u4, u5};
  double dp, dm;
  weno5_face<double, false>(ud, (double)inv, dp, dm);
  return make_float2((float)dp, (float)dm);
}

// True when the smoothness indicators of a stencil differ by more than a
// factor 1e3, i.e. the stencil straddles a kink.  Used by the FP32 form to
// recompute such values in FP64.
template <typename T>
__device__ __forceinline__ bool weno5_is_kink(T v1, T v2, T v3, T v4, T v5) {
  T t = v1 - T(2) * v2 + v3, u = v1 - T(4) * v2 + T(3) * v3;
  const T S1 = T(13.0 / 12.0) * (t * t) + T(0.25) * (u * u);
  t = v2 - T(2) * v3 + v4;
  u = v2 - v4;
  const T S2 = T(13.0 / 12.0) * (t * t) + T(0.25) * (u * u);
  t = v3 - T(2) * v4 + v5;
  u = T(3) * v3 - T(4) * v4 + v5;
  const T S3 = T(13.0 / 12.0) * (t * t) + T(0.25) * (u * u);
  const T mx = vmax(vmax(S1, S2), S3), mn = vmin(vmin(S1, S2), S3);
  const T scale = vmax(vmax(vmax(v1 * v1, v2 * v2), vmax(v3 * v3, v4 * v4)), v5 * v5);
  return mx > T(1e3) * mn + T(1e-4) * scale;
}

}  // namespace lsmgpu
