// stage_launch.h -- type-erased arguments of the fused stage kernels.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace lsmgpu {

struct StageArgs {
  void* out;
  const void* phi_s;
  const void* phi_n;
  const void* aux[3];
  void* rhs_out;
  double* partials;
  Box gb;
  FillBox fb;
  FillBox dom;
  unsigned bc_mask;
  double inv[3];
  double dx_sq;
  const double* dt_dev;
  double dt;
  int rk_kind;
  int use_phi0;
  int fp64_policy;  // kFp64Kinks | kFp64Sign | kStochRound (FP32 form)
  unsigned sr_seed; // nonzero: stochastic rounding of the output (FP32)
  const double* defo_tab;  // kStageDeformation (see StageParams)
  int defo_off[3];
  const double* g_dev;
  // the stage input's ghost cells may be written (set by the drivers, whose
  // arrays these are): the face-shared kinds then store the boundary values
  // of bc_mask into phi_s's ghost cells and read them as stored
  int ghosts_writable;
};

// tile of the stage kernels: TX x TY cells per block, TZ planes per block
// (build-time settings; TX is one warp)
#ifndef LSMGPU_STAGE_TY
#define LSMGPU_STAGE_TY 8
#endif
#ifndef LSMGPU_STAGE_TZ
#define LSMGPU_STAGE_TZ 16
#endif
constexpr int kStageTX = 32, kStageTY = LSMGPU_STAGE_TY, kStageTZ = LSMGPU_STAGE_TZ;

inline int stage_blocks(const FillBox& fb) {
  const int gx = (fb.n(0) + kStageTX - 1) / kStageTX;
  const int gy = (fb.n(1) + kStageTY - 1) / kStageTY;
  const int gz = (fb.n(2) + kStageTZ - 1) / kStageTZ;
  return gx * gy * gz;
}

// kind: StageKind; prec: 8 (FP64) or 4 (FP32)
cudaError_t launch_stage_strict(int kind, int prec, const StageArgs& a,
                                cudaStream_t st);
cudaError_t launch_stage_fast(int kind, int prec, const StageArgs& a,
                              cudaStream_t st);

}  // namespace lsmgpu
