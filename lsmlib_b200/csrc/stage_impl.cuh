// stage_impl.cuh -- instantiation of the fused stage kernels for one
// arithmetic mode.  Included once by stage_strict.cu (STAGE_FAST = false,
// built with --fmad=false) and once by stage_fast.cu (STAGE_FAST = true, FMA).
#include <algorithm>

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
  for (int d = 0; d < 3; d++) {
    p.inv[d] = (T)a.inv[d];
    p.fk[d] = face_const<T>(p.inv[d]);
  }
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

#ifndef LSMGPU_STAGE_PAIRS
#define LSMGPU_STAGE_PAIRS 1
#endif

// The boundary values of a.bc_mask can be stored in phi_s's ghost cells:
// the caller allows it, and every axis with a boundary kind has at least 3
// domain cells (so no ghost value depends on another ghost cell).
bool ghosts_storable(const StageArgs& a) {
  if (!a.ghosts_writable) return false;
  for (int d = 0; d < 3; d++) {
    const unsigned face_bits = 3u << (2 * d);
    const bool any = (a.bc_mask & (face_bits | face_bits << 8 | face_bits << 16)) != 0u;
    if (any && a.dom.n(d) < 3) return false;
  }
  return true;
}

// The boundary values of a.bc_mask into phi_s's ghost cells: the planes of
// the fill box, and the z faces its stencils reach (about 4 cells per
// thread of a z ghost plane).
template <typename T>
void launch_face_ghosts(const StageArgs& a, cudaStream_t st) {
  const int zchunks = (int)std::min<long>(
      4096, ((long)a.dom.n(0) * a.dom.n(1) + 4 * kFaceGhostThreads - 1) /
                (4 * kFaceGhostThreads));
  const long groups = (a.fb.n(2) + kGhostPlanes - 1) / kGhostPlanes;
  const long blocks = groups * face_ghost_xy_blocks(a.dom.n(0), a.dom.n(1)) + 6L * zchunks;
  k_face_ghosts<T><<<(unsigned)blocks, kFaceGhostThreads, 0, st>>>(
      (T*)a.phi_s, a.gb, a.dom, a.bc_mask, a.fb.lo[2], a.fb.hi[2], zchunks);
  ++launch_counter();
}

// The pair kernels take the stage: offsets fit 32 bits, and the ghost cells
// are stored (no boundary kind, or k_face_ghosts can write them first).
bool pairs_apply(const StageArgs& a) {
  const bool small = a.gb.sz() * (long)a.gb.n[2] < (1L << 31);   // 32-bit offsets
  return small && (a.bc_mask == 0u || ghosts_storable(a));
}

// One kind: a two-cells-per-thread kernel where it applies (FMA or FP32
// arithmetic; the face-shared kernel for the two-sided kinds, the one-sided
// pair kernel for the upwind kinds) and pairs_apply; else one cell per
// thread with the boundary values generated on the fly.  All cover TX x TY
// x TZ cells per block, so the grid (and the per-block CFL partials) are
// the same.
template <typename T, int KIND>
void launch_kind(dim3 grid, const StageArgs& a, const StageParams<T>& p, cudaStream_t st) {
  constexpr int TX = kStageTX, TY = kStageTY, TZ = kStageTZ;
  if constexpr (LSMGPU_STAGE_PAIRS && UseFaces<T, KIND, STAGE_FAST, TX>::value) {
    if (pairs_apply(a)) {
      StageParams<T> q = p;
      if (a.bc_mask != 0u) {
        launch_face_ghosts<T>(a, st);
        q.bc_mask = 0u;
      }
      const dim3 blk(TX / 2, TY, 1);
      if constexpr (sizeof(T) == 4) {
        if (p.fp64_policy & kFp64Kinks) {
          k_stage_pairs<T, KIND, true, TX, TY, TZ><<<grid, blk, 0, st>>>(q);
          return;
        }
      }
      k_stage_pairs<T, KIND, false, TX, TY, TZ><<<grid, blk, 0, st>>>(q);
      return;
    }
  }
  if constexpr (LSMGPU_STAGE_PAIRS && UsePairsUp<T, KIND, STAGE_FAST, TX>::value) {
    if (pairs_apply(a)) {
      StageParams<T> q = p;
      if (a.bc_mask != 0u) {
        launch_face_ghosts<T>(a, st);
        q.bc_mask = 0u;
      }
      const dim3 blk(TX / 2, TY, 1);
      if constexpr (sizeof(T) == 4) {
        if (p.fp64_policy & kFp64Kinks) {
          k_stage_pairs_up<T, KIND, true, TX, TY, TZ><<<grid, blk, 0, st>>>(q);
          return;
        }
      }
      k_stage_pairs_up<T, KIND, false, TX, TY, TZ><<<grid, blk, 0, st>>>(q);
      return;
    }
  }
  k_stage<T, KIND, STAGE_FAST, TX, TY, TZ><<<grid, dim3(TX, TY, 1), 0, st>>>(p);
}

template <typename T>
cudaError_t launch_t(int kind, const StageArgs& a, cudaStream_t st) {
  constexpr int TX = kStageTX, TY = kStageTY, TZ = kStageTZ;
  const FillBox& fb = a.fb;
  dim3 grid((fb.n(0) + TX - 1) / TX, (fb.n(1) + TY - 1) / TY,
            (fb.n(2) + TZ - 1) / TZ);
  const StageParams<T> p = to_params<T>(a);
  switch (kind) {
    case kStageAdvect: launch_kind<T, kStageAdvect>(grid, a, p, st); break;
    case kStageNormal: launch_kind<T, kStageNormal>(grid, a, p, st); break;
    case kStageReinit: launch_kind<T, kStageReinit>(grid, a, p, st); break;
    case kStageDeformation: launch_kind<T, kStageDeformation>(grid, a, p, st); break;
    case kStageNormalRhs: launch_kind<T, kStageNormalRhs>(grid, a, p, st); break;
    default:
      return cudaErrorInvalidValue;
  }
  ++launch_counter();
  return cudaGetLastError();
}

#ifdef STAGE_BAND_FN
// the FP64 band form of one upwind kind: FP32 launch for the tiles flagged 0,
// FP64 launch for those flagged 1, each also writing the other precision
template <int KIND>
cudaError_t band_kind(dim3 grid, const StageArgs& a32, const StageArgs& a64,
                      const unsigned char* tile_fp64, cudaStream_t st, cudaStream_t side,
                      cudaEvent_t ev[2]) {
  constexpr int TX = kStageTX, TY = kStageTY, TZ = kStageTZ;
  static_assert(UsePairsUp<float, KIND, STAGE_FAST, TX>::value &&
                    UsePairsUp<double, KIND, STAGE_FAST, TX>::value,
                "the band form runs the two-cells-per-thread upwind kernels");
  if (!pairs_apply(a32) || !pairs_apply(a64)) return cudaErrorNotSupported;
  StageParams<float> q32 = to_params<float>(a32);
  StageParams<double> q64 = to_params<double>(a64);
  if (a32.bc_mask != 0u) {
    launch_face_ghosts<float>(a32, st);
    launch_face_ghosts<double>(a64, st);
    q32.bc_mask = q64.bc_mask = 0u;
  }
  q32.tile_fp64 = q64.tile_fp64 = tile_fp64;
  q32.tile_want = 0u;
  q64.tile_want = 1u;
  q32.out_alt = a64.out;
  q64.out_alt = a32.out;
  const dim3 blk(TX / 2, TY, 1);
  cudaError_t e;
  if ((e = cudaEventRecord(ev[0], st)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(side, ev[0], 0)) != cudaSuccess)
    return e;
  k_stage_pairs_up<double, KIND, false, TX, TY, TZ, true><<<grid, blk, 0, side>>>(q64);
  if (q32.fp64_policy & kFp64Kinks)
    k_stage_pairs_up<float, KIND, true, TX, TY, TZ, true><<<grid, blk, 0, st>>>(q32);
  else
    k_stage_pairs_up<float, KIND, false, TX, TY, TZ, true><<<grid, blk, 0, st>>>(q32);
  launch_counter() += 2;
  if ((e = cudaEventRecord(ev[1], side)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(st, ev[1], 0)) != cudaSuccess)
    return e;
  return cudaGetLastError();
}
#endif

}  // namespace

#ifdef STAGE_BAND_FN
cudaError_t STAGE_BAND_FN(int kind, const StageArgs& a32, const StageArgs& a64,
                          const unsigned char* tile_fp64, cudaStream_t st, cudaStream_t side,
                          cudaEvent_t ev[2]) {
  constexpr int TX = kStageTX, TY = kStageTY, TZ = kStageTZ;
  const FillBox& fb = a32.fb;
  if (fb.n(0) < 1 || fb.n(1) < 1 || fb.n(2) < 1) return cudaSuccess;
  const dim3 grid((fb.n(0) + TX - 1) / TX, (fb.n(1) + TY - 1) / TY,
                  (fb.n(2) + TZ - 1) / TZ);
  switch (kind) {
    case kStageDeformation:
      return band_kind<kStageDeformation>(grid, a32, a64, tile_fp64, st, side, ev);
    default: return cudaErrorInvalidValue;
  }
}
#endif

cudaError_t STAGE_LAUNCH_FN(int kind, int prec, const StageArgs& a,
                            cudaStream_t st) {
  if (a.fb.n(0) < 1 || a.fb.n(1) < 1 || a.fb.n(2) < 1) return cudaSuccess;
  return prec == 8 ? launch_t<double>(kind, a, st) : launch_t<float>(kind, a, st);
}

}  // namespace lsmgpu
