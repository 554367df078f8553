// common.cuh -- device-side building blocks shared by every lsmgpu kernel.
//
// Arrays follow the reference's Fortran convention: element (i,j,k) of an
// array whose ghost box is [ilo:ihi]x[jlo:jhi]x[klo:khi] is stored at
// (i-ilo) + nx*((j-jlo) + ny*(k-klo))  (doc/doxygen/users_guide/
// lsmlib_toolbox_package.dox, "NOTES").  A Grid3 carries a base pointer
// pre-shifted by the lower bounds so that the offset of (i,j,k) is
// i + sy*j + sz*k.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lsmgpu {

// Precision constants of the reference build (configure.ac:264-272).
template <typename T> struct Consts;
template <> struct Consts<double> {
  static constexpr double tiny = 1.0e-99;   // @tiny_nonzero_number@ (FP64)
  static constexpr double zero_tol = 1.0e-11;  // @lsmlib_zero_tol@ (FP64)
};
template <> struct Consts<float> {
  static constexpr float tiny = 1.0e-35f;   // --enable-float build
  static constexpr float zero_tol = 1.0e-5f;
};

// Host-side description of one array: lower corner and extents of its ghost
// box.  Passed by value to kernels.
struct Box {
  int lo[3];
  int n[3];
  __host__ __device__ long sy() const { return (long)n[0]; }
  __host__ __device__ long sz() const { return (long)n[0] * (long)n[1]; }
  __host__ __device__ long count() const {
    return (long)n[0] * (long)n[1] * (long)n[2];
  }
  __host__ __device__ int hi(int d) const { return lo[d] + n[d] - 1; }
};

template <typename T>
struct Grid3 {
  T* base;   // points at (0,0,0) in index space (may lie outside the array)
  long sy, sz;
  __host__ __device__ T& operator()(int i, int j, int k) const {
    return base[(long)i + sy * (long)j + sz * (long)k];
  }
  __host__ __device__ T* ptr(int i, int j, int k) const {
    return base + ((long)i + sy * (long)j + sz * (long)k);
  }
  __host__ __device__ long stride(int d) const {
    return d == 0 ? 1L : (d == 1 ? sy : sz);
  }
};

template <typename T>
__host__ __device__ inline Grid3<T> make_grid(T* p, const Box& b) {
  Grid3<T> g;
  g.sy = b.sy();
  g.sz = b.sz();
  g.base = p - ((long)b.lo[0] + g.sy * (long)b.lo[1] + g.sz * (long)b.lo[2]);
  return g;
}

// Fill box (cells a routine writes), inclusive bounds.
struct FillBox {
  int lo[3], hi[3];
  __host__ __device__ int n(int d) const { return hi[d] - lo[d] + 1; }
  __host__ __device__ long count() const {
    return (long)n(0) * (long)n(1) * (long)n(2);
  }
};

// Fortran MAX/MIN on reals: a > b ? a : b (equal to the reference for
// non-NaN data).
template <typename T> __device__ __forceinline__ T fmax2(T a, T b) {
  return a > b ? a : b;
}
template <typename T> __device__ __forceinline__ T fmin2(T a, T b) {
  return a < b ? a : b;
}
__device__ __forceinline__ double fabsT(double x) { return fabs(x); }
__device__ __forceinline__ float fabsT(float x) { return fabsf(x); }
__device__ __forceinline__ double sqrtT(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrtT(float x) { return sqrtf(x); }

// Stochastic rounding of FP32 state updates.  Round-to-nearest drops every
// update smaller than half an ulp of phi in the same direction, so over the
// thousands of stage updates of a run (reinitialization near its steady
// state in particular) the FP32 state drifts from the FP64 one.  Rounding
// up with probability (x - down(x)) / ulp makes the stored value unbiased,
// E[round(x)] = x, and the drift a random walk (Connolly, Higham & Mary,
// SIAM J. Sci. Comput., 2021; Paxton et al., Mon. Weather Rev., 2022).
// The random integer comes from a counter-based hash of the cell offset and
// a per-launch seed, so a run is reproducible.

// 32-bit integer finaliser ("lowbias32", C. Wellons, hash-prospector)
__host__ __device__ __forceinline__ unsigned sr_hash(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// x rounded to FP32 stochastically with the low 29 bits of r: adding a
// uniform integer below 2^29 to the magnitude bits of the FP64 value and
// truncating those 29 bits (the FP64 significand carries 29 bits more than
// the FP32 one) rounds up with exactly the probability above; the truncated
// value converts to FP32 without further rounding (normal FP32 range).
__device__ __forceinline__ float sr_float(double x, unsigned r) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  const unsigned long long sign = b & 0x8000000000000000ull;
  unsigned long long mag = (b ^ sign) + (unsigned long long)(r & 0x1fffffffu);
  mag &= ~0x1fffffffull;
  return (float)__longlong_as_double((long long)(mag | sign));
}

// Status word that kernels may raise (never trap): bit 0 = bad argument seen
// on the device, bit 1 = a bounded wait gave up.
enum DeviceStatus : unsigned { kDevOk = 0u, kDevBadArg = 1u, kDevTimeout = 2u };

}  // namespace lsmgpu
