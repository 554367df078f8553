// stage_impl.cuh -- instantiation of the fused stage kernels for one
// arithmetic mode.  Included once by stage_strict.cu (STAGE_FAST = false,
// built with --fmad=false) and once by stage_fast.cu (STAGE_FAST = true, FMA).
#include "launch.h"
#include "stage.cuh"
#include "stage_launch.h"

namespace lsmgpu {
namespace {

template <typename T>
StageParams<T> to_params(const StageArgs& a) {
  StageParams<T> p;
  p.out = (T*)a.out;
  p.phi_s = (const T*)a.phi_s;
  p.phi_n = (const T*)a.phi_n;
  p.aux0 = (const T*)a.aux[0];
  p.aux1 = (const T*)a.aux[1];
  p.aux2 = (const T*)a.aux[2];
  p.rhs_out = (T*)a.rhs_out;
  p.partials = a.partials;
  p.gb = a.gb;
  p.fb = a.fb;
  p.dom = a.dom;
  p.bc_mask = a.bc_mask;
  for (int d = 0; d < 3; d++) p.inv[d] = (T)a.inv[d];
  p.dx_sq = (T)a.dx_sq;
  p.dt_dev = a.dt_dev;
  p.dt = a.dt;
  p.rk_kind = a.rk_kind;
  p.use_phi0 = a.use_phi0;
  p.fp64_policy = a.fp64_policy;
  p.sr_seed = a.sr_seed;
  p.defo_tab = a.defo_tab;
  for (int d = 0; d < 3; d++) p.defo_off[d] = a.defo_off[d];
  p.g_dev = a.g_dev;
  return p;
}

template <typename T>
cudaError_t launch_t(int kind, const StageArgs& a, cudaStream_t st) {
  constexpr int TX = kStageTX, TY = kStageTY, TZ = kStageTZ;
  const FillBox& fb = a.fb;
  dim3 grid((fb.n(0) + TX - 1) / TX, (fb.n(1) + TY - 1) / TY,
            (fb.n(2) + TZ - 1) / TZ);
  dim3 blk(TX, TY, 1);
  const StageParams<T> p = to_params<T>(a);
  switch (kind) {
    case kStageAdvect:
      k_stage<T, kStageAdvect, STAGE_FAST, TX, TY, TZ><<<grid, blk, 0, st>>>(p);
      break;
    case kStageNormal:
      k_stage<T, kStageNormal, STAGE_FAST, TX, TY, TZ><<<grid, blk, 0, st>>>(p);
      break;
    case kStageReinit:
      k_stage<T, kStageReinit, STAGE_FAST, TX, TY, TZ><<<grid, blk, 0, st>>>(p);
      break;
    case kStageDeformation:
      k_stage<T, kStageDeformation, STAGE_FAST, TX, TY, TZ><<<grid, blk, 0, st>>>(p);
      break;
    case kStageNormalRhs:
      k_stage<T, kStageNormalRhs, STAGE_FAST, TX, TY, TZ><<<grid, blk, 0, st>>>(p);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  ++launch_counter();
  return cudaGetLastError();
}

}  // namespace

cudaError_t STAGE_LAUNCH_FN(int kind, int prec, const StageArgs& a,
                            cudaStream_t st) {
  if (a.fb.n(0) < 1 || a.fb.n(1) < 1 || a.fb.n(2) < 1) return cudaSuccess;
  return prec == 8 ? launch_t<double>(kind, a, st) : launch_t<float>(kind, a, st);
}

}  // namespace lsmgpu
