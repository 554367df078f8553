// launch.h -- host-side launchers of the lsmgpu kernels (C++ only, no CUDA
// syntax), shared by the C ABI layer and the integrators.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace lsmgpu {

// Number of kernels this library has launched (host-side count).
unsigned long long& launch_counter();

// ---- drop-in toolbox kernels (reference expression order, no FMA) -------
// T is double (FP64) or float (FP32); ``prec`` is sizeof(T).
cudaError_t launch_hj_plus_minus(int scheme, int prec, void* const out_plus[3],
                                 const Box& gplus, void* const out_minus[3],
                                 const Box& gminus, const void* phi,
                                 const Box& gphi, const FillBox& fb,
                                 const double inv[3], cudaStream_t st);
cudaError_t launch_hj_upwind(int scheme, int prec, void* const out[3],
                             const Box& gout, const void* phi, const Box& gphi,
                             const void* const vel[3], const Box& gvel,
                             const FillBox& fb, const double inv[3],
                             cudaStream_t st);
cudaError_t launch_fill(int prec, void* p, long count, double value,
                        cudaStream_t st);
cudaError_t launch_add_advection(int prec, void* rhs, const Box& grhs,
                                 const void* const grad[3], const Box& ggrad,
                                 const void* const vel[3], const Box& gvel,
                                 const FillBox& fb, cudaStream_t st);
// vel_n == nullptr selects the constant-speed variant with speed ``vn_const``
cudaError_t launch_add_normal(int prec, void* rhs, const Box& grhs,
                              const void* const gp[3], const Box& gplus,
                              const void* const gm[3], const Box& gminus,
                              const void* vel_n, const Box& gvel,
                              double vn_const, const FillBox& fb,
                              cudaStream_t st);
cudaError_t launch_reinit_rhs(int prec, void* rhs, const Box& grhs,
                              const void* phi, const Box& gphi,
                              const void* phi0, const Box& gphi0,
                              const void* const gp[3], const Box& gplus,
                              const void* const gm[3], const Box& gminus,
                              const FillBox& fb, double dx_sq, int use_phi0,
                              cudaStream_t st);
cudaError_t launch_field_ext_rhs(int prec, void* rhs, const Box& grhs,
                                 const void* phi, const Box& gphi,
                                 const void* const gs[3], const Box& ggs,
                                 const void* const nrm[3], const Box& gnrm,
                                 const FillBox& fb, double cutoff,
                                 cudaStream_t st);
cudaError_t launch_signed_normal(int prec, void* const nrm[3], const Box& gnrm,
                                 const void* const grad[3], const Box& ggrad,
                                 const void* phi, const Box& gphi,
                                 const FillBox& fb, double dx_sq,
                                 cudaStream_t st);
// kind: 1 = u1 = u + dt*L, 22 = TVD-RK2 stage 2, 32 = TVD-RK3 stage 2,
// 33 = TVD-RK3 stage 3.  ``us`` is the previous stage (unused for kind 1).
// ``dt_dev`` (device) overrides ``dt`` when non-null.
cudaError_t launch_rk(int prec, int kind, void* out, const Box& gout,
                      const void* us, const Box& gus, const void* uc,
                      const Box& guc, const void* rhs, const Box& grhs,
                      const FillBox& fb, double dt, const double* dt_dev,
                      cudaStream_t st, unsigned sr_seed = 0u);
// face 0..5; copy = 0 linear extrapolation, 1 copy extrapolation
cudaError_t launch_bc(int prec, int copy, void* phi, const Box& gphi,
                      const FillBox& fb, int face, cudaStream_t st);

// ---- reductions: partial maxima, then a one-block finish that writes the
// result (max, or dt = cfl/(max + tiny)) to ``result_dev`` (double). ------
enum ReduceKind { kRedMaxNormDiff = 0, kRedAdvectionDt = 1, kRedNormalDt = 2 };
int reduce_partials_needed(const FillBox& ib);
// ``partials`` must hold reduce_partials_needed(ib) doubles.
cudaError_t launch_max_norm_diff(int prec, const void* f1, const Box& g1,
                                 const void* f2, const Box& g2,
                                 const FillBox& ib, double* partials,
                                 double* result_dev, cudaStream_t st);
cudaError_t launch_stable_advection_dt(int prec, const void* const vel[3],
                                       const Box& gvel, const FillBox& ib,
                                       const double inv[3], double cfl,
                                       double* partials, double* result_dev,
                                       cudaStream_t st);
// vel_n == nullptr: constant speed ``vn_const``
cudaError_t launch_stable_normal_dt(int prec, const void* vel_n,
                                    const Box& gvel, double vn_const,
                                    const void* const gp[3], const Box& gplus,
                                    const void* const gm[3], const Box& gminus,
                                    const FillBox& ib, const double inv[3],
                                    double max_dx_sq, double cfl,
                                    double* partials, double* result_dev,
                                    cudaStream_t st);

}  // namespace lsmgpu
