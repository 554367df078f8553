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
// One stage of kStageDeformation (velocity evaluated in the kernel, so both
// precisions have it) in the FP64 band form, fast arithmetic: a32 and a64 name the same stage over the FP32
// arrays and their FP64 copies; tile_fp64[tile] (tiles as in stage_blocks,
// x fastest) = 1 computes the tile in FP64, 0 in FP32.  Both launches write
// every output cell in both precisions.  cudaErrorNotSupported when the
// two-cells-per-thread kernels do not apply (arrays of 2^31 or more cells,
// or boundary values that cannot be stored in the ghost cells).
// The FP64 launch runs on `side` (forked from st after the ghost fills by
// event ev[0], joined back by ev[1]), so that the FP64 tiles run beside the
// FP32 launch instead of after it.
cudaError_t launch_stage_band(int kind, const StageArgs& a32, const StageArgs& a64,
                              const unsigned char* tile_fp64, cudaStream_t st,
                              cudaStream_t side, cudaEvent_t ev[2]);

}  // namespace lsmgpu
