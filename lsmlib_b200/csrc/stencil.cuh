// stencil.cuh -- one-sided ENO/WENO derivatives along one axis.
//
// All functions take q = pointer to the cell, s = element stride of the axis
// and inv = 1/dx of the axis.  The undivided differences are formed on the
// fly from phi, with the same doubles the reference stores in its D1/D2/D3
// scratch arrays (lsm3dComputeDn, lsm_spatial_derivatives3d.f.in:49-176):
//   D1(m) = phi(m) - phi(m-1)          (face m-1/2)
//   D2(m) = -(D1(m) - D1(m+1))         (the negation turns an exact zero
//                                        into -0.0, as the reference does)
//   D3(m) = D2(m) - D2(m-1)
// "Strict" forms repeat the reference's floating-point expression order; the
// translation unit that instantiates them is compiled with --fmad=false, so
// with IEEE division and square root they are bit-identical to the reference.
#pragma once
#include "common.cuh"

namespace lsmgpu {

template <typename T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

template <typename T>
__device__ __forceinline__ T D1(const T* q, long s, int m) {
  return ld(q + m * s) - ld(q + (m - 1) * s);
}
template <typename T>
__device__ __forceinline__ T D2(const T* q, long s, int m) {
  return -(D1(q, s, m) - D1(q, s, m + 1));
}
template <typename T>
__device__ __forceinline__ T D3(const T* q, long s, int m) {
  return D2(q, s, m) - D2(q, s, m - 1);
}

// HJ-WENO5 reconstruction, reference expression order
// (lsm_spatial_derivatives3d.f.in:1292-1323).
template <typename T>
__device__ __forceinline__ T weno5_strict(T v1, T v2, T v3, T v4, T v5) {
  const T one_third = T(1.0) / T(3.0);
  const T seven_sixths = T(7.0) / T(6.0);
  const T eleven_sixths = T(11.0) / T(6.0);
  const T one_sixth = T(1.0) / T(6.0);
  const T five_sixths = T(5.0) / T(6.0);
  const T thirteen_twelfths = T(13.0) / T(12.0);
  const T one_fourth = T(0.25);
  T m = fmax2(v1 * v1, v2 * v2);
  m = fmax2(m, v3 * v3);
  m = fmax2(m, v4 * v4);
  m = fmax2(m, v5 * v5);
  const T eps = T(1e-6) * m + Consts<T>::tiny;
  const T p1 = one_third * v1 - seven_sixths * v2 + eleven_sixths * v3;
  const T p2 = -(one_sixth * v2) + five_sixths * v3 + one_third * v4;
  const T p3 = one_third * v3 + five_sixths * v4 - one_sixth * v5;
  T t = v1 - T(2.0) * v2 + v3;
  T u = v1 - T(4.0) * v2 + T(3.0) * v3;
  const T S1 = thirteen_twelfths * (t * t) + one_fourth * (u * u);
  t = v2 - T(2.0) * v3 + v4;
  u = v2 - v4;
  const T S2 = thirteen_twelfths * (t * t) + one_fourth * (u * u);
  t = v3 - T(2.0) * v4 + v5;
  u = T(3.0) * v3 - T(4.0) * v4 + v5;
  const T S3 = thirteen_twelfths * (t * t) + one_fourth * (u * u);
  t = S1 + eps;
  T a1 = T(0.1) / (t * t);
  t = S2 + eps;
  T a2 = T(0.6) / (t * t);
  t = S3 + eps;
  T a3 = T(0.3) / (t * t);
  const T inv_sum_a = T(1.0) / (a1 + a2 + a3);
  a1 = a1 * inv_sum_a;
  a2 = a2 * inv_sum_a;
  a3 = a3 * inv_sum_a;
  return a1 * p1 + a2 * p2 + a3 * p3;
}

// ENO1 / ENO2 / ENO3 one-sided values, reference expression order
// (lsm_spatial_derivatives3d.f.in:299-300, :520-535, :842-896).
template <typename T>
__device__ __forceinline__ T eno2_plus(const T* q, long s, T inv) {
  const T half = T(0.5);
  const T a = D2(q, s, 0), b = D2(q, s, 1);
  return (fabsT(a) < fabsT(b)) ? (D1(q, s, 1) - half * a) * inv
                               : (D1(q, s, 1) - half * b) * inv;
}
template <typename T>
__device__ __forceinline__ T eno2_minus(const T* q, long s, T inv) {
  const T half = T(0.5);
  const T a = D2(q, s, -1), b = D2(q, s, 0);
  return (fabsT(a) < fabsT(b)) ? (D1(q, s, 0) + half * a) * inv
                               : (D1(q, s, 0) + half * b) * inv;
}
template <typename T>
__device__ __forceinline__ T eno3_plus(const T* q, long s, T inv) {
  const T half = T(0.5), third = T(1.0) / T(3.0), sixth = T(1.0) / T(6.0);
  T r = D1(q, s, 1);
  if (fabsT(D2(q, s, 0)) < fabsT(D2(q, s, 1))) {
    r = r - half * D2(q, s, 0);
    const T a = D3(q, s, 0), b = D3(q, s, 1);
    r = (fabsT(a) < fabsT(b)) ? r - sixth * a : r - sixth * b;
  } else {
    r = r - half * D2(q, s, 1);
    const T a = D3(q, s, 1), b = D3(q, s, 2);
    r = (fabsT(a) < fabsT(b)) ? r + third * a : r + third * b;
  }
  return r * inv;
}
template <typename T>
__device__ __forceinline__ T eno3_minus(const T* q, long s, T inv) {
  const T half = T(0.5), third = T(1.0) / T(3.0), sixth = T(1.0) / T(6.0);
  T r = D1(q, s, 0);
  if (fabsT(D2(q, s, -1)) < fabsT(D2(q, s, 0))) {
    r = r + half * D2(q, s, -1);
    const T a = D3(q, s, -1), b = D3(q, s, 0);
    r = (fabsT(a) < fabsT(b)) ? r + third * a : r + third * b;
  } else {
    r = r + half * D2(q, s, 0);
    const T a = D3(q, s, 0), b = D3(q, s, 1);
    r = (fabsT(a) < fabsT(b)) ? r - sixth * a : r - sixth * b;
  }
  return r * inv;
}

enum Scheme { kENO1 = 1, kENO2 = 2, kENO3 = 3, kWENO5 = 5 };

// Ghost width each scheme reads on either side of a fill-box cell.
__host__ __device__ constexpr int scheme_width(int scheme) {
  return scheme == kWENO5 ? 3 : scheme;
}

template <int SCHEME, typename T>
__device__ __forceinline__ T plus_strict(const T* q, long s, T inv) {
  if (SCHEME == kENO1) return D1(q, s, 1) * inv;
  if (SCHEME == kENO2) return eno2_plus(q, s, inv);
  if (SCHEME == kENO3) return eno3_plus(q, s, inv);
  return weno5_strict(D1(q, s, 3) * inv, D1(q, s, 2) * inv, D1(q, s, 1) * inv,
                      D1(q, s, 0) * inv, D1(q, s, -1) * inv);
}
template <int SCHEME, typename T>
__device__ __forceinline__ T minus_strict(const T* q, long s, T inv) {
  if (SCHEME == kENO1) return D1(q, s, 0) * inv;
  if (SCHEME == kENO2) return eno2_minus(q, s, inv);
  if (SCHEME == kENO3) return eno3_minus(q, s, inv);
  return weno5_strict(D1(q, s, -2) * inv, D1(q, s, -1) * inv, D1(q, s, 0) * inv,
                      D1(q, s, 1) * inv, D1(q, s, 2) * inv);
}

}  // namespace lsmgpu
