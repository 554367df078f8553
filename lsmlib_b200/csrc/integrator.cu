// integrator.cu -- fused TVD-RK3 time stepping (extension API, Part 2 of
// include/lsmgpu/lsmgpu.h).
//
// A workspace owns the stage buffers of one grid (phi^(1), phi^(2), the stage
// RHS, phi0 for the reinitialization sign, deformation sine tables, device scalars
// dt and t, and the CFL partial maxima).  The drivers reproduce the call
// order of the reference's integrators
//   LevelSetFunctionIntegrator::advanceLevelSetEqnUsingTVDRK3
//     (LevelSetFunctionIntegrator.cc:1319-1510; dt from computeStableDt,
//     :345-587; reinitialization every interval steps, :658-697)
//   ReinitializationAlgorithm::reinitializeLevelSetFunctions
//     (ReinitializationAlgorithm.cc:177-330; dt = cfl * min dx, :216)
// with one fused kernel per Runge-Kutta stage.  dt and t live on the device,
// so a whole run is launched without a host synchronisation.
#include <cmath>
#include <cstring>
#include <string>

#include "capi_common.h"
#include "launch.h"
#include "stage.cuh"
#include "stage_launch.h"

using namespace lsmgpu;

// z-slabs of the host-array driver's copies (see lsmgpu_normal_tvdrk3_host)
#ifndef LSMGPU_HOST_SLABS
#define LSMGPU_HOST_SLABS 4
#endif
constexpr int kHostSlabs = LSMGPU_HOST_SLABS;
// speed buffers of queued host-array calls: up to kMaxSpeedBufs, as many as
// fit in 1 GiB (at least 2)
constexpr int kMaxSpeedBufs = 8;

struct lsmgpu_workspace {
  Box gb;
  int prec;
  size_t bytes;
  void* phi1 = nullptr;
  void* phi2 = nullptr;
  void* rhs = nullptr;
  void* phi0 = nullptr;
  // lsmgpu_normal_tvdrk3_host: device copies of the host level set and of
  // the speed (nspeed buffers, taken in turn by queued calls), the streams
  // of the slab copies to and from the host and of the queued calls' speed
  // uploads, and per slab: copied in, final stage done, copied out; per
  // speed buffer: last read, upload done (created on first use)
  void* dphi = nullptr;
  void* dF[kMaxSpeedBufs] = {};
  int nspeed = 0;
  cudaStream_t copy_stream = nullptr;       // host -> device
  cudaStream_t copy_stream_out = nullptr;   // device -> host
  cudaStream_t copy_stream_F = nullptr;     // host -> device, queued calls' speed
  cudaEvent_t slab_ev[2 * kHostSlabs] = {};  // [q] in, [kHostSlabs + q] final stage
  cudaEvent_t out_ev[kHostSlabs] = {};
  cudaEvent_t F_ev[kMaxSpeedBufs] = {};
  cudaEvent_t Fin_ev[kMaxSpeedBufs] = {};
  // per call (ring of nspeed): its level set uploaded; and the last queued
  // call that ran a reinitialization (-1: none)
  cudaEvent_t up_ev[kMaxSpeedBufs] = {};
  long long last_reinit_call = -1;
  cudaEvent_t start_ev = nullptr;
  int host_async = 0;       // lsmgpu_workspace_set_host_async
  int host_pending = 0;     // a queued host call has not been waited for
  unsigned host_calls = 0;
  double* defo_tab = nullptr;   // deformation sine tables (see stage.cuh)
  size_t defo_len = 0;
  double* scal = nullptr;   // device scalars (kDt, kT, kDtLast, kG0..kG0+2)
  double* partials = nullptr;
  int npart = 0;
  unsigned bc_mask = 0x3fu;
  int fp64_policy = kFp64Sign | kStochRound;  // FP32 workspaces only
  // FP64 band form (kFp64Band): FP64 copies of phi, phi^(1) and phi^(2)
  // (created on first use), the per-tile flags (those within band_cells
  // cells of the interface, then the same widened by one tile), and the
  // band half-width in cells
  double* band64[3] = {nullptr, nullptr, nullptr};
  unsigned char* band_flags = nullptr;
  int band_tiles = 0;
  double band_cells = 16.0;
  int band_widen = 1;   // tiles added around the flagged ones (0 or 1)
  // the stream of the FP64 tiles' launches (high priority, so that their
  // blocks are placed before the FP32 launch's), and its fork/join events
  cudaStream_t band_stream = nullptr;
  cudaEvent_t band_ev[2] = {nullptr, nullptr};
  unsigned sr_launches = 0;  // stochastic-rounding seeds drawn so far
  unsigned long long steps = 0;
};

namespace {

// device scalars of a workspace: dt, t, the dt of the last step, and g of
// the deformation field at t, t + dt, t + dt/2 (the three stage times)
enum { kDt = 0, kT = 1, kDtLast = 2, kG0 = 3, kNumScal = 8 };

__device__ __forceinline__ double gmax(double m, double v) { return v > m ? v : m; }

// dt = cfl / (max + tiny) (lsm_utilities3d.f.in:322, :445), optionally
// clipped so that t + dt does not pass t_end
__global__ void k_dt_finish(const double* partials, int np, double cfl,
                            double tiny, double* scal, double t_end) {
  __shared__ double red[8];
  double m = -1.0;
  for (int t = threadIdx.x; t < np; t += blockDim.x) m = gmax(m, partials[t]);
  for (int o = 16; o > 0; o >>= 1) m = gmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = gmax(m, red[w]);
    m = gmax(red[0], m);
    double dt = cfl / (m + tiny);
    if (t_end > 0.0 && scal[kT] + dt > t_end) dt = t_end - scal[kT];
    scal[kDt] = dt;
  }
}

__global__ void k_set_dt(double* scal, double dt) { scal[kDt] = dt; }
__global__ void k_advance_t(double* scal) {
  scal[kT] = scal[kT] + scal[kDt];
  scal[kDtLast] = scal[kDt];
}

// LeVeque's 3D deformation field (deformation_velocity, stage.cuh) at cell
// centres x_i = x_lo + (i + 1/2) dx, with g(t) = cos(pi t / period).  The
// sines of every fill-box coordinate are tabulated once per call and g once
// per stage time, so the stage kernels and the CFL reduction evaluate the
// field without velocity arrays; both are computed here, in the translation
// unit without FMA contraction, from the same expressions as before the
// tabulation.
__global__ void k_deform_tables(double* tab, FillBox fb, double x0, double y0,
                                double z0, double dx, double dy, double dz) {
  const int n0 = fb.n(0), n1 = fb.n(1), n2 = fb.n(2);
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  double x;
  double* out;
  int n;
  if (q < n0) {
    x = x0 + (fb.lo[0] + q + 0.5) * dx; out = tab + q; n = n0;
  } else if (q < n0 + n1) {
    x = y0 + (fb.lo[1] + (q - n0) + 0.5) * dy; out = tab + 2 * n0 + (q - n0); n = n1;
  } else if (q < n0 + n1 + n2) {
    x = z0 + (fb.lo[2] + (q - n0 - n1) + 0.5) * dz;
    out = tab + 2 * n0 + 2 * n1 + (q - n0 - n1); n = n2;
  } else {
    return;
  }
  out[0] = sin(M_PI * x);
  out[n] = sin(2.0 * M_PI * x);
}

__device__ __forceinline__ double deform_g(const double* scal, double c, double period) {
  const double t = scal[kT] + c * scal[kDt];
  return cos(M_PI * t / period);
}

// g at the three stage times t, t + dt, t + dt/2 (after this step's dt)
__global__ void k_deform_g(double* scal, double period) {
  const double c[3] = {0.0, 1.0, 0.5};
  if (threadIdx.x < 3) scal[kG0 + threadIdx.x] = deform_g(scal, c[threadIdx.x], period);
}

// the CFL reduction of the deformation field at time t (FP64), over the
// velocity components rounded to the working precision T as the stage
// kernels see them
template <typename T>
__global__ void k_deform_partials(const double* tab, FillBox fb, const double* scal,
                                  double period, double ix, double iy, double iz,
                                  double* partials) {
  const double g = deform_g(scal, 0.0, period);
  const int n0 = fb.n(0), n1 = fb.n(1), n2 = fb.n(2);
  double m = -1.0;
  const long n = fb.count();
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const int a = (int)(t % n0);
    const long r = t / n0;
    const int b = (int)(r % n1), c = (int)(r / n1);
    DeformSines s;
    s.sx = tab[a]; s.s2x = tab[n0 + a];
    s.sy = tab[2 * n0 + b]; s.s2y = tab[2 * n0 + n1 + b];
    s.sz = tab[2 * n0 + 2 * n1 + c]; s.s2z = tab[2 * n0 + 2 * n1 + n2 + c];
    T u, v, w;
    deformation_velocity(s, g, u, v, w);
    const double h = fabs((double)u) * ix + fabs((double)v) * iy + fabs((double)w) * iz;
    m = gmax(m, h);
  }
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) m = gmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = gmax(m, red[w]);
    partials[blockIdx.x] = gmax(red[0], m);
  }
}

// the CFL reduction of velocity arrays (FP64)
template <typename T>
__global__ void k_adv_partials(const T* vx, const T* vy, const T* vz, Box gb,
                               FillBox fb, double ix, double iy, double iz,
                               double* partials) {
  double m = -1.0;
  const long n = fb.count();
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const int i = fb.lo[0] + (int)(t % fb.n(0));
    const long r = t / fb.n(0);
    const int j = fb.lo[1] + (int)(r % fb.n(1));
    const int k = fb.lo[2] + (int)(r / fb.n(1));
    const long o = (long)(i - gb.lo[0]) + gb.sy() * (j - gb.lo[1]) +
                   gb.sz() * (k - gb.lo[2]);
    const double u = fabs((double)vx[o]) * ix + fabs((double)vy[o]) * iy +
                     fabs((double)vz[o]) * iz;
    m = gmax(m, u);
  }
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) m = gmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = gmax(m, red[w]);
    partials[blockIdx.x] = gmax(red[0], m);
  }
}

constexpr int kAdvRedBlocks = 1184;

// FP64 band form.  The FP64 copy of the caller's FP32 level set is kept
// between calls; a cell whose copy no longer rounds to the caller's value
// (first use, or phi changed by the caller) is reloaded from phi.
__global__ void k_band_sync(const float* phi, double* copy, long n) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const float v = phi[t];
    if (!((float)copy[t] == v)) copy[t] = (double)v;
  }
}

// flag[tile] = 1 when some cell of the tile (stage tiles of kStageTX x
// kStageTY x kStageTZ cells, numbered x fastest) has |phi| < thr
__global__ void __launch_bounds__(256) k_band_tiles(const float* phi, Box gb, FillBox fb,
                                                    float thr, unsigned char* flag) {
  const int x0 = fb.lo[0] + blockIdx.x * kStageTX, y0 = fb.lo[1] + blockIdx.y * kStageTY,
            z0 = fb.lo[2] + blockIdx.z * kStageTZ;
  const int x = x0 + (threadIdx.x & (kStageTX - 1));
  int near = 0;
  if (x <= fb.hi[0]) {
    for (int r = threadIdx.x / kStageTX; r < kStageTY * kStageTZ; r += blockDim.x / kStageTX) {
      const int y = y0 + r % kStageTY, z = z0 + r / kStageTY;
      if (y > fb.hi[1] || z > fb.hi[2]) continue;
      const long o = (long)(x - gb.lo[0]) + gb.sy() * (y - gb.lo[1]) + gb.sz() * (z - gb.lo[2]);
      near |= fabsf(phi[o]) < thr;
    }
  }
  near = __syncthreads_or(near);
  if (threadIdx.x == 0)
    flag[blockIdx.x + gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z)] =
        (unsigned char)(near != 0);
}

// out[tile] = 1 when the tile or one of its 26 neighbours has in[] = 1
__global__ void k_band_widen(const unsigned char* in, unsigned char* out, int gx, int gy,
                             int gz) {
  const long n = (long)gx * gy * gz;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const int x = (int)(t % gx), y = (int)((t / gx) % gy), z = (int)(t / ((long)gx * gy));
    unsigned char f = 0;
    for (int c = max(z - 1, 0); c <= min(z + 1, gz - 1); c++)
      for (int b = max(y - 1, 0); b <= min(y + 1, gy - 1); b++)
        for (int a = max(x - 1, 0); a <= min(x + 1, gx - 1); a++)
          f |= in[a + (long)gx * (b + (long)gy * c)];
    out[t] = f;
  }
}

// A boundary mask (stage.cuh: bit f linear, 8+f copy, 16+f periodic) is
// usable by the multi-step drivers when every face has exactly one kind and
// periodic faces come in lo/hi pairs.
bool bc_mask_complete(unsigned m) {
  for (int f = 0; f < 6; f++) {
    const int kinds = ((m >> f) & 1u) + ((m >> (8 + f)) & 1u) + ((m >> (16 + f)) & 1u);
    if (kinds != 1) return false;
  }
  for (int d = 0; d < 3; d++)
    if (((m >> (16 + 2 * d)) & 1u) != ((m >> (17 + 2 * d)) & 1u)) return false;
  return true;
}

bool ws_ok(lsmgpu_workspace* ws, const char* R) {
  if (!ws) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null workspace");
    return false;
  }
  return true;
}

bool fb_in(const Box& gb, const FillBox& fb, int w, const char* R) {
  return covers(gb, fb, w, "phi", R);
}

void* ws_alloc(size_t bytes, const char* R) {
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error(LSMGPU_ERR_ALLOC, std::string(R) + ": cudaMalloc failed");
    return nullptr;
  }
  return p;
}

// seed of the next stochastically rounded launch of an FP32 workspace (0 when
// its policy rounds to nearest)
unsigned next_sr_seed(lsmgpu_workspace* ws) {
  if (!ws || ws->prec != 4 || !(ws->fp64_policy & kStochRound)) return 0u;
  return sr_hash(++ws->sr_launches * 0x9e3779b9u) | 1u;
}

cudaError_t stage(int kind, int prec, StageArgs a, cudaStream_t st,
                  lsmgpu_workspace* ws = nullptr) {
  a.sr_seed = next_sr_seed(ws);
  return fp_mode() == LSMGPU_FP_FAST ? launch_stage_fast(kind, prec, a, st)
                                     : launch_stage_strict(kind, prec, a, st);
}

// The band form runs the two-cells-per-thread upwind kernels, which need
// offsets below 2^31 and the boundary values stored in the ghost cells
// (3 domain cells on every axis with a boundary kind); elsewhere the plain
// FP32 form runs.
bool band_applies(const lsmgpu_workspace* ws, const FillBox& f) {
  if (ws->gb.count() >= (1L << 31)) return false;
  for (int d = 0; d < 3; d++) {
    const unsigned face_bits = 3u << (2 * d);
    const bool any = (ws->bc_mask & (face_bits | face_bits << 8 | face_bits << 16)) != 0u;
    if (any && f.n(d) < 3) return false;
  }
  return true;
}

// FP64 band form: the FP64 copies and flag arrays for fill box f, and the
// FP64 copy of phi brought in line with the caller's phi
bool band_setup(lsmgpu_workspace* ws, const void* phi, const FillBox& f, cudaStream_t st,
                const char* R) {
  const size_t bytes64 = (size_t)ws->gb.count() * sizeof(double);
  for (int q = 0; q < 3; q++) {
    if (ws->band64[q]) continue;
    if (!(ws->band64[q] = (double*)ws_alloc(bytes64, R))) return false;
    // the copy of phi starts as NaN, so that k_band_sync loads every cell
    if (!cuda_ok(cudaMemsetAsync(ws->band64[q], q == 0 ? 0xff : 0, bytes64, st), R))
      return false;
  }
  if (!ws->band_stream) {
    int lo = 0, hi = 0;
    if (!cuda_ok(cudaDeviceGetStreamPriorityRange(&lo, &hi), R) ||
        !cuda_ok(cudaStreamCreateWithPriority(&ws->band_stream, cudaStreamNonBlocking, hi), R) ||
        !cuda_ok(cudaEventCreateWithFlags(&ws->band_ev[0], cudaEventDisableTiming), R) ||
        !cuda_ok(cudaEventCreateWithFlags(&ws->band_ev[1], cudaEventDisableTiming), R))
      return false;
  }
  const int tiles = stage_blocks(f);
  if (ws->band_tiles < tiles) {
    if (ws->band_flags) cudaFree(ws->band_flags);
    ws->band_tiles = 0;
    if (!(ws->band_flags = (unsigned char*)ws_alloc(2 * (size_t)tiles, R))) return false;
    ws->band_tiles = tiles;
  }
  // a grid-stride pass: four 256-thread blocks per SM of a B200 (148 SMs)
  k_band_sync<<<4 * 148, 256, 0, st>>>((const float*)phi, ws->band64[0], ws->gb.count());
  ++launch_counter();
  return cuda_ok(cudaGetLastError(), R);
}

// the tiles of fill box f computed in FP64 this step: within band_cells cells
// (|phi| < band_cells * min dx) of the interface, widened by one tile
void band_flags(lsmgpu_workspace* ws, const void* phi, const FillBox& f, const double dx[3],
                cudaStream_t st) {
  const dim3 tg((f.n(0) + kStageTX - 1) / kStageTX, (f.n(1) + kStageTY - 1) / kStageTY,
                (f.n(2) + kStageTZ - 1) / kStageTZ);
  const int tiles = (int)(tg.x * tg.y * tg.z);
  double mn = dx[0] < dx[1] ? dx[0] : dx[1];
  mn = mn < dx[2] ? mn : dx[2];
  // without widening the tiles are flagged straight into the second half
  k_band_tiles<<<tg, 256, 0, st>>>((const float*)phi, ws->gb, f, (float)(ws->band_cells * mn),
                                   ws->band_flags + (ws->band_widen ? 0 : tiles));
  ++launch_counter();
  if (ws->band_widen) {
    k_band_widen<<<(tiles + 255) / 256, 256, 0, st>>>(ws->band_flags, ws->band_flags + tiles,
                                                       (int)tg.x, (int)tg.y, (int)tg.z);
    ++launch_counter();
  }
}

// one stage in the FP64 band form: a names the FP32 arrays (phi or the
// workspace's), the FP64 launch takes their copies
cudaError_t band_stage(int kind, lsmgpu_workspace* ws, const void* phi, StageArgs a,
                       cudaStream_t st) {
  auto copy_of = [&](const void* p) -> double* {
    if (p == phi) return ws->band64[0];
    if (p == ws->phi1) return ws->band64[1];
    if (p == ws->phi2) return ws->band64[2];
    return nullptr;
  };
  a.sr_seed = next_sr_seed(ws);
  StageArgs b = a;
  b.out = copy_of(a.out);
  b.phi_s = copy_of(a.phi_s);
  b.phi_n = copy_of(a.phi_n);
  b.fp64_policy = 0;
  b.sr_seed = 0u;
  if (!b.out || !b.phi_s || !b.phi_n) return cudaErrorInvalidValue;
  return launch_stage_band(kind, a, b, ws->band_flags + stage_blocks(a.fb), st,
                           ws->band_stream, ws->band_ev);
}

StageArgs base_args(lsmgpu_workspace* ws, const FillBox& fb, const double dx[3]) {
  StageArgs a;
  memset(&a, 0, sizeof a);
  a.gb = ws->gb;
  a.fb = fb;
  a.dom = fb;
  a.bc_mask = ws->bc_mask;
  for (int d = 0; d < 3; d++) a.inv[d] = 1.0 / dx[d];
  double m = dx[0] > dx[1] ? dx[0] : dx[1];
  m = m > dx[2] ? m : dx[2];
  a.dx_sq = m * m;
  a.dt_dev = ws->scal + kDt;
  a.fp64_policy = ws->prec == 4 ? ws->fp64_policy : 0;
  // the drivers' stage inputs are phi and the workspace arrays: their ghost
  // cells take the boundary values before each stage, as the reference's
  // boundary module fills them (edge and corner ghosts are not written)
  a.ghosts_writable = 1;
  return a;
}

// One TVD-RK3 reinitialization pseudo-step of phi (in place) with dt = dtr.
bool reinit_step(lsmgpu_workspace* ws, void* phi, const FillBox& fb,
                 const double dx[3], double dtr, int use0, cudaStream_t st,
                 const char* R) {
  StageArgs a = base_args(ws, fb, dx);
  a.dt_dev = nullptr;
  a.dt = dtr;
  a.use_phi0 = use0;
  a.aux[0] = ws->phi0;
  a.out = ws->phi1; a.phi_s = phi; a.phi_n = phi; a.rk_kind = 1;
  if (!cuda_ok(stage(kStageReinit, ws->prec, a, st, ws), R)) return false;
  a.out = ws->phi2; a.phi_s = ws->phi1; a.rk_kind = 32;
  if (!cuda_ok(stage(kStageReinit, ws->prec, a, st, ws), R)) return false;
  a.out = phi; a.phi_s = ws->phi2; a.rk_kind = 33;
  return cuda_ok(stage(kStageReinit, ws->prec, a, st, ws), R);
}

bool reinit_run(lsmgpu_workspace* ws, void* phi, const FillBox& fb,
                const double dx[3], double cfl, int iters, int use0,
                cudaStream_t st, const char* R) {
  if (iters <= 0) return true;
  if (use0 == 1) {
    if (!ws->phi0 && !(ws->phi0 = ws_alloc(ws->bytes, R))) return false;
    if (!cuda_ok(cudaMemcpyAsync(ws->phi0, phi, ws->bytes,
                                 cudaMemcpyDeviceToDevice, st),
                 R))
      return false;
  }
  // ReinitializationAlgorithm.cc:211-216: dt = cfl * min(dx)
  double mn = dx[0] < dx[1] ? dx[0] : dx[1];
  mn = mn < dx[2] ? mn : dx[2];
  const double dtr = cfl * mn;
  for (int it = 0; it < iters; it++)
    if (!reinit_step(ws, phi, fb, dx, dtr, use0, st, R)) return false;
  return true;
}

FillBox fb6(const int* f) {
  FillBox b;
  b.lo[0] = f[0]; b.hi[0] = f[1];
  b.lo[1] = f[2]; b.hi[1] = f[3];
  b.lo[2] = f[4]; b.hi[2] = f[5];
  return b;
}

bool common_checks(lsmgpu_workspace* ws, const void* phi, const int* fb,
                   const double* dx, const char* R, FillBox* out) {
  clear_error();
  if (!ws_ok(ws, R)) return false;
  if (!phi || !fb || !dx) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return false;
  }
  *out = fb6(fb);
  if (out->n(0) < 2 || out->n(1) < 2 || out->n(2) < 2) {
    set_error(LSMGPU_ERR_INVALID_BOX,
              std::string(R) + ": the fill box needs two cells per axis");
    return false;
  }
  if (!fb_in(ws->gb, *out, 3, R)) return false;
  if (!(dx[0] > 0 && dx[1] > 0 && dx[2] > 0)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": dx must be positive");
    return false;
  }
  if (!bc_mask_complete(ws->bc_mask)) {
    set_error(LSMGPU_ERR_INVALID_VALUE,
              std::string(R) + ": multi-step drivers need one generated "
                               "boundary kind on every face (periodic in pairs)");
    return false;
  }
  return true;
}

}  // namespace

extern "C" {

int lsmgpu_workspace_create(lsmgpu_workspace** out, const int gb[6],
                            int precision) {
  const char* R = "lsmgpu_workspace_create";
  clear_error();
  if (!out || !gb) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  *out = nullptr;
  if (precision != 8 && precision != 4) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": precision is 8 or 4");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  lsmgpu_workspace* ws = new lsmgpu_workspace();
  ws->gb = box_from(&gb[0], &gb[1], &gb[2], &gb[3], &gb[4], &gb[5]);
  if (!box_valid(ws->gb, "phi", R)) {
    delete ws;
    return LSMGPU_ERR_INVALID_BOX;
  }
  ws->prec = precision;
  ws->bytes = (size_t)ws->gb.count() * (size_t)precision;
  ws->npart = kAdvRedBlocks;
  FillBox whole;
  for (int d = 0; d < 3; d++) { whole.lo[d] = ws->gb.lo[d]; whole.hi[d] = ws->gb.hi(d); }
  if (stage_blocks(whole) > ws->npart) ws->npart = stage_blocks(whole);
  if (!(ws->phi1 = ws_alloc(ws->bytes, R)) || !(ws->phi2 = ws_alloc(ws->bytes, R)) ||
      !(ws->rhs = ws_alloc(ws->bytes, R)) ||
      !(ws->scal = (double*)ws_alloc(sizeof(double) * kNumScal, R)) ||
      !(ws->partials = (double*)ws_alloc(sizeof(double) * ws->npart, R))) {
    lsmgpu_workspace_destroy(ws);
    return LSMGPU_ERR_ALLOC;
  }
  cudaMemset(ws->scal, 0, sizeof(double) * kNumScal);
  // the stage buffers are only ever read inside the fill box, but start them
  // from zero so that no uninitialised memory is ever read by a caller
  cudaMemset(ws->phi1, 0, ws->bytes);
  cudaMemset(ws->phi2, 0, ws->bytes);
  cudaMemset(ws->rhs, 0, ws->bytes);
  if (!cuda_ok(cudaDeviceSynchronize(), R)) {
    lsmgpu_workspace_destroy(ws);
    return LSMGPU_ERR_CUDA;
  }
  *out = ws;
  return LSMGPU_SUCCESS;
}

int lsmgpu_workspace_destroy(lsmgpu_workspace* ws) {
  if (!ws) return LSMGPU_SUCCESS;
  if (ws->host_pending) lsmgpu_workspace_sync(ws);
  void* ps[] = {ws->phi1,      ws->phi2,      ws->rhs,       ws->phi0,      ws->defo_tab,
                ws->scal,      ws->partials,  ws->dphi,      ws->band64[0], ws->band64[1],
                ws->band64[2], ws->band_flags};
  for (void* p : ps)
    if (p) cudaFree(p);
  for (void* p : ws->dF)
    if (p) cudaFree(p);
  for (cudaEvent_t e : ws->Fin_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ws->up_ev)
    if (e) cudaEventDestroy(e);
  if (ws->copy_stream_F) cudaStreamDestroy(ws->copy_stream_F);
  for (cudaEvent_t e : ws->slab_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ws->out_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ws->F_ev)
    if (e) cudaEventDestroy(e);
  if (ws->start_ev) cudaEventDestroy(ws->start_ev);
  for (cudaEvent_t e : ws->band_ev)
    if (e) cudaEventDestroy(e);
  if (ws->band_stream) cudaStreamDestroy(ws->band_stream);
  if (ws->copy_stream) cudaStreamDestroy(ws->copy_stream);
  if (ws->copy_stream_out) cudaStreamDestroy(ws->copy_stream_out);
  delete ws;
  return LSMGPU_SUCCESS;
}

int lsmgpu_workspace_set_host_async(lsmgpu_workspace* ws, int on) {
  if (!ws_ok(ws, "lsmgpu_workspace_set_host_async")) return LSMGPU_ERR_NULL_POINTER;
  if (!on && ws->host_pending) {
    const int rc = lsmgpu_workspace_sync(ws);
    if (rc != LSMGPU_SUCCESS) return rc;
  }
  ws->host_async = on ? 1 : 0;
  return LSMGPU_SUCCESS;
}

int lsmgpu_workspace_sync(lsmgpu_workspace* ws) {
  const char* R = "lsmgpu_workspace_sync";
  if (!ws_ok(ws, R)) return LSMGPU_ERR_NULL_POINTER;
  if (!ws->host_pending) return LSMGPU_SUCCESS;
  ws->host_pending = 0;
  // the copies back to the host are the last work of a host call; the
  // speed buffers' events close its kernels
  if (!cuda_ok(cudaStreamSynchronize(ws->copy_stream_out), R) ||
      !cuda_ok(cudaStreamSynchronize(ws->copy_stream), R) ||
      !cuda_ok(cudaStreamSynchronize(ws->copy_stream_F), R))
    return LSMGPU_ERR_CUDA;
  for (cudaEvent_t e : ws->F_ev)
    if (!cuda_ok(cudaEventSynchronize(e), R)) return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

int lsmgpu_workspace_set_bc(lsmgpu_workspace* ws, unsigned linear_faces_mask) {
  // bits 0-5 linear, 8-13 copy, 16-21 periodic (face f = x-lo .. z-hi)
  if (!ws_ok(ws, "lsmgpu_workspace_set_bc")) return LSMGPU_ERR_NULL_POINTER;
  ws->bc_mask = linear_faces_mask & (kBcLinear | kBcCopy | kBcPeriodic);
  return LSMGPU_SUCCESS;
}

int lsmgpu_workspace_set_fp64_policy(lsmgpu_workspace* ws, int policy) {
  // bit 0: WENO5 kink stencils in FP64; bit 1: reinitialization sign in FP64;
  // bit 2: stochastic rounding of the FP32 stage outputs; bit 3: the tiles
  // near the interface in FP64 (deformation driver, fast mode)
  if (!ws_ok(ws, "lsmgpu_workspace_set_fp64_policy")) return LSMGPU_ERR_NULL_POINTER;
  if (policy & ~(kFp64Kinks | kFp64Sign | kStochRound | kFp64Band)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, "lsmgpu_workspace_set_fp64_policy: unknown bits");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  ws->fp64_policy = policy;
  return LSMGPU_SUCCESS;
}

int lsmgpu_workspace_set_fp64_band(lsmgpu_workspace* ws, double cells, int widen) {
  if (!ws_ok(ws, "lsmgpu_workspace_set_fp64_band")) return LSMGPU_ERR_NULL_POINTER;
  if (!(cells >= 0.0) || (widen != 0 && widen != 1)) {
    set_error(LSMGPU_ERR_INVALID_VALUE,
              "lsmgpu_workspace_set_fp64_band: cells >= 0 and widen 0 or 1");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  ws->band_cells = cells;
  ws->band_widen = widen;
  return LSMGPU_SUCCESS;
}

int lsmgpu_workspace_set_time(lsmgpu_workspace* ws, double t) {
  if (!ws_ok(ws, "lsmgpu_workspace_set_time")) return LSMGPU_ERR_NULL_POINTER;
  double v[2] = {0.0, t};
  return cuda_ok(cudaMemcpy(ws->scal, v, sizeof v, cudaMemcpyHostToDevice),
                 "lsmgpu_workspace_set_time")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}

// host copy of t and of the dt of the last step (waits for the stream)
int lsmgpu_workspace_get_time(lsmgpu_workspace* ws, double* t, double* dt_last) {
  if (!ws_ok(ws, "lsmgpu_workspace_get_time")) return LSMGPU_ERR_NULL_POINTER;
  double v[kNumScal];
  cudaStream_t st = cur_stream();
  if (!cuda_ok(cudaMemcpyAsync(v, ws->scal, sizeof v, cudaMemcpyDeviceToHost, st),
               "lsmgpu_workspace_get_time") ||
      !cuda_ok(cudaStreamSynchronize(st), "lsmgpu_workspace_get_time"))
    return LSMGPU_ERR_CUDA;
  if (t) *t = v[kT];
  if (dt_last) *dt_last = v[kDtLast];
  return LSMGPU_SUCCESS;
}

const double* lsmgpu_workspace_device_scalars(lsmgpu_workspace* ws) {
  return ws ? ws->scal : nullptr;
}

// One fused stage on caller-owned device arrays (all with ghost box gb).
int lsmgpu_lse_stage(int kind, int precision, void* out, const void* phi_s,
                     const void* phi_n, const void* aux0, const void* aux1,
                     const void* aux2, const int gb[6], const int fb[6],
                     const int dom[6], unsigned bc_mask, const double dx[3],
                     const double* dt_dev, double dt, int rk_kind,
                     int use_phi0) {
  const char* R = "lsmgpu_lse_stage";
  clear_error();
  if (!out || !phi_s || !gb || !fb || !dx || (rk_kind != 1 && !phi_n) ||
      (kind == kStageAdvect && (!aux0 || !aux1 || !aux2)) ||
      (kind == kStageNormal && !aux0) ||
      (kind == kStageReinit && use_phi0 == 1 && !aux0)) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  if (kind < kStageAdvect || kind > kStageReinit || (precision != 8 && precision != 4) ||
      (rk_kind != 1 && rk_kind != 22 && rk_kind != 32 && rk_kind != 33)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": bad kind/precision/rk");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  const Box g = box_from(&gb[0], &gb[1], &gb[2], &gb[3], &gb[4], &gb[5]);
  const FillBox f = fb6(fb);
  if (f.n(0) < 1 || f.n(1) < 1 || f.n(2) < 1) return LSMGPU_SUCCESS;
  if (!box_valid(g, "phi", R) || !covers(g, f, 3, "phi", R))
    return LSMGPU_ERR_INVALID_BOX;
  StageArgs a;
  memset(&a, 0, sizeof a);
  a.gb = g;
  a.fb = f;
  a.bc_mask = bc_mask & (kBcLinear | kBcCopy | kBcPeriodic);
  for (int d = 0; d < 3; d++)
    if (((a.bc_mask >> (16 + 2 * d)) & 1u) != ((a.bc_mask >> (17 + 2 * d)) & 1u)) {
      set_error(LSMGPU_ERR_INVALID_VALUE,
                std::string(R) + ": periodic faces come in lo/hi pairs");
      return LSMGPU_ERR_INVALID_VALUE;
    }
  a.dom = dom ? fb6(dom) : f;
  if (a.bc_mask) {
    for (int d = 0; d < 3; d++)
      if (a.dom.lo[d] > f.lo[d] || a.dom.hi[d] < f.hi[d] ||
          a.dom.hi[d] - a.dom.lo[d] < 1 || a.dom.lo[d] < g.lo[d] ||
          a.dom.hi[d] > g.hi(d)) {
        set_error(LSMGPU_ERR_INVALID_BOX,
                  std::string(R) + ": domain box must contain the fill box, "
                                   "lie in the ghost box and span 2 cells");
        return LSMGPU_ERR_INVALID_BOX;
      }
  }
  a.out = out; a.phi_s = phi_s; a.phi_n = phi_n;
  a.aux[0] = aux0; a.aux[1] = aux1; a.aux[2] = aux2;
  for (int d = 0; d < 3; d++) a.inv[d] = 1.0 / dx[d];
  double m = dx[0] > dx[1] ? dx[0] : dx[1];
  m = m > dx[2] ? m : dx[2];
  a.dx_sq = m * m;
  a.dt_dev = dt_dev;
  a.dt = dt;
  a.rk_kind = rk_kind;
  a.use_phi0 = use_phi0;
  a.fp64_policy = precision == 4 ? kFp64Sign : 0;
  cudaStream_t st = cur_stream();
  if (!cuda_ok(stage(kind, precision, a, st), R)) return LSMGPU_ERR_CUDA;
  if (sync_mode() && !cuda_ok(cudaStreamSynchronize(st), R)) return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

// Linear-extrapolation ghost fill of all six faces in the reference's order
// (lsm_boundary_conditions.c:227-293, case 9).
int lsmgpu_fill_ghosts_linear(void* phi, int precision, const int gb[6],
                              const int fb[6]) {
  const char* R = "lsmgpu_fill_ghosts_linear";
  clear_error();
  if (!phi || !gb || !fb) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  const Box g = box_from(&gb[0], &gb[1], &gb[2], &gb[3], &gb[4], &gb[5]);
  const FillBox f = fb6(fb);
  if (!box_valid(g, "phi", R) || !covers(g, f, 0, "phi", R)) return LSMGPU_ERR_INVALID_BOX;
  if (f.n(0) < 2 || f.n(1) < 2 || f.n(2) < 2) {
    set_error(LSMGPU_ERR_INVALID_BOX, std::string(R) + ": fill box too thin");
    return LSMGPU_ERR_INVALID_BOX;
  }
  cudaStream_t st = cur_stream();
  for (int face = 0; face < 6; face++)
    if (!cuda_ok(launch_bc(precision, 0, phi, g, f, face, st), R)) return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

// TVD-RK3 steps under an external velocity field (device arrays with the
// workspace ghost box).  dt_fixed > 0: constant dt; otherwise the CFL dt of
// LSM3D_COMPUTE_STABLE_ADVECTION_DT every step (clipped at t_end > 0).
int lsmgpu_advect_tvdrk3(lsmgpu_workspace* ws, void* phi, const void* vx,
                         const void* vy, const void* vz, const int fb[6],
                         const double dx[3], double cfl, double dt_fixed,
                         double t_end, int nsteps) {
  const char* R = "lsmgpu_advect_tvdrk3";
  FillBox f;
  if (!common_checks(ws, phi, fb, dx, R, &f)) return lsmgpu_peek_last_error();
  if (!vx || !vy || !vz) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null velocity");
    return LSMGPU_ERR_NULL_POINTER;
  }
  cudaStream_t st = cur_stream();
  const void* vel[3] = {vx, vy, vz};
  const double tiny = ws->prec == 8 ? Consts<double>::tiny : (double)Consts<float>::tiny;
  for (int s = 0; s < nsteps; s++) {
    if (dt_fixed > 0) {
      k_set_dt<<<1, 1, 0, st>>>(ws->scal, dt_fixed);
    } else {
      const double inv[3] = {1.0 / dx[0], 1.0 / dx[1], 1.0 / dx[2]};
      if (ws->prec == 8)
        k_adv_partials<double><<<kAdvRedBlocks, 256, 0, st>>>(
            (const double*)vx, (const double*)vy, (const double*)vz, ws->gb, f,
            inv[0], inv[1], inv[2], ws->partials);
      else
        k_adv_partials<float><<<kAdvRedBlocks, 256, 0, st>>>(
            (const float*)vx, (const float*)vy, (const float*)vz, ws->gb, f,
            inv[0], inv[1], inv[2], ws->partials);
      ++launch_counter();
      k_dt_finish<<<1, 256, 0, st>>>(ws->partials, kAdvRedBlocks, cfl, tiny,
                                     ws->scal, t_end);
    }
    ++launch_counter();
    StageArgs a = base_args(ws, f, dx);
    for (int d = 0; d < 3; d++) a.aux[d] = vel[d];
    a.out = ws->phi1; a.phi_s = phi; a.phi_n = phi; a.rk_kind = 1;
    if (!cuda_ok(stage(kStageAdvect, ws->prec, a, st, ws), R)) return LSMGPU_ERR_CUDA;
    a.out = ws->phi2; a.phi_s = ws->phi1; a.rk_kind = 32;
    if (!cuda_ok(stage(kStageAdvect, ws->prec, a, st, ws), R)) return LSMGPU_ERR_CUDA;
    a.out = phi; a.phi_s = ws->phi2; a.rk_kind = 33;
    if (!cuda_ok(stage(kStageAdvect, ws->prec, a, st, ws), R)) return LSMGPU_ERR_CUDA;
    k_advance_t<<<1, 1, 0, st>>>(ws->scal);
    ++launch_counter();
    ws->steps++;
  }
  if (!cuda_ok(cudaGetLastError(), R)) return LSMGPU_ERR_CUDA;
  if (sync_mode() && !cuda_ok(cudaStreamSynchronize(st), R)) return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

// TVD-RK3 steps under the deformation field of LeVeque (period ``period``),
// velocity re-evaluated at t, t+dt, t+dt/2 for the three stages
// (LevelSetFunctionIntegrator.cc:1332, :1404, :1476); CFL dt every step from
// the velocity at t, clipped at t_end.  x_lo is the lower corner of the
// domain; cell centres sit at x_lo + (i + 1/2) dx.
int lsmgpu_deformation_tvdrk3(lsmgpu_workspace* ws, void* phi, const int fb[6],
                              const double dx[3], const double x_lo[3],
                              double period, double cfl, double t_end,
                              int nsteps) {
  const char* R = "lsmgpu_deformation_tvdrk3";
  FillBox f;
  if (!common_checks(ws, phi, fb, dx, R, &f)) return lsmgpu_peek_last_error();
  if (!x_lo || !(period > 0)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": bad x_lo/period");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  // sine tables of the fill-box coordinates (sin(pi x), sin(2 pi x) per axis)
  const size_t len = 2 * ((size_t)f.n(0) + f.n(1) + f.n(2));
  if (ws->defo_len < len) {
    if (ws->defo_tab) cudaFree(ws->defo_tab);
    ws->defo_len = 0;
    if (!(ws->defo_tab = (double*)ws_alloc(len * sizeof(double), R))) return LSMGPU_ERR_ALLOC;
    ws->defo_len = len;
  }
  cudaStream_t st = cur_stream();
  const int nt = f.n(0) + f.n(1) + f.n(2);
  k_deform_tables<<<(nt + 127) / 128, 128, 0, st>>>(ws->defo_tab, f, x_lo[0], x_lo[1],
                                                    x_lo[2], dx[0], dx[1], dx[2]);
  ++launch_counter();
  // FP64 band form: the tiles near the interface in FP64, with the dt of the
  // FP64 velocity, as an FP64 workspace computes them
  const bool band = ws->prec == 4 && (ws->fp64_policy & kFp64Band) &&
                    fp_mode() == LSMGPU_FP_FAST && band_applies(ws, f);
  if (band && !band_setup(ws, phi, f, st, R)) return lsmgpu_peek_last_error();
  const double tiny =
      ws->prec == 8 || band ? Consts<double>::tiny : (double)Consts<float>::tiny;
  const double inv[3] = {1.0 / dx[0], 1.0 / dx[1], 1.0 / dx[2]};
  auto run = [&](StageArgs& a) {
    return band ? band_stage(kStageDeformation, ws, phi, a, st)
                : stage(kStageDeformation, ws->prec, a, st, ws);
  };
  for (int s = 0; s < nsteps; s++) {
    // dt from the field at t (the stage-1 field)
    if (ws->prec == 8 || band)
      k_deform_partials<double><<<kAdvRedBlocks, 256, 0, st>>>(
          ws->defo_tab, f, ws->scal, period, inv[0], inv[1], inv[2], ws->partials);
    else
      k_deform_partials<float><<<kAdvRedBlocks, 256, 0, st>>>(
          ws->defo_tab, f, ws->scal, period, inv[0], inv[1], inv[2], ws->partials);
    k_dt_finish<<<1, 256, 0, st>>>(ws->partials, kAdvRedBlocks, cfl, tiny, ws->scal,
                                   t_end);
    k_deform_g<<<1, 32, 0, st>>>(ws->scal, period);
    launch_counter() += 3;
    StageArgs a = base_args(ws, f, dx);
    a.defo_tab = ws->defo_tab;
    a.defo_off[0] = 0;
    a.defo_off[1] = 2 * f.n(0);
    a.defo_off[2] = 2 * (f.n(0) + f.n(1));
    if (band) band_flags(ws, phi, f, dx, st);
    // velocity at t, t + dt, t + dt/2 for the three stages
    a.g_dev = ws->scal + kG0;
    a.out = ws->phi1; a.phi_s = phi; a.phi_n = phi; a.rk_kind = 1;
    if (!cuda_ok(run(a), R)) return LSMGPU_ERR_CUDA;
    a.g_dev = ws->scal + kG0 + 1;
    a.out = ws->phi2; a.phi_s = ws->phi1; a.rk_kind = 32;
    if (!cuda_ok(run(a), R)) return LSMGPU_ERR_CUDA;
    a.g_dev = ws->scal + kG0 + 2;
    a.out = phi; a.phi_s = ws->phi2; a.rk_kind = 33;
    if (!cuda_ok(run(a), R)) return LSMGPU_ERR_CUDA;
    k_advance_t<<<1, 1, 0, st>>>(ws->scal);
    ++launch_counter();
    ws->steps++;
  }
  if (!cuda_ok(cudaGetLastError(), R)) return LSMGPU_ERR_CUDA;
  if (sync_mode() && !cuda_ok(cudaStreamSynchronize(st), R)) return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

// TVD-RK3 steps of phi_t + F |grad phi| = 0 with a normal-speed array F and
// the CFL dt of LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT every step; after every
// reinit_interval-th step (counted from step0) reinit_iters reinitialization
// pseudo-steps.
int lsmgpu_normal_tvdrk3(lsmgpu_workspace* ws, void* phi, const void* F,
                         const int fb[6], const double dx[3], double cfl,
                         int nsteps, int step0, int reinit_interval,
                         int reinit_iters, int use_phi0_for_sgn) {
  const char* R = "lsmgpu_normal_tvdrk3";
  FillBox f;
  if (!common_checks(ws, phi, fb, dx, R, &f)) return lsmgpu_peek_last_error();
  if (!F) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null speed");
    return LSMGPU_ERR_NULL_POINTER;
  }
  cudaStream_t st = cur_stream();
  const double tiny = ws->prec == 8 ? Consts<double>::tiny : (double)Consts<float>::tiny;
  const int nblk = stage_blocks(f);
  for (int s = 0; s < nsteps; s++) {
    StageArgs a = base_args(ws, f, dx);
    a.aux[0] = F;
    // WENO5 +- of phi^n once: L(phi^n) for stage 1 and the CFL maxima
    a.rhs_out = ws->rhs; a.partials = ws->partials; a.phi_s = phi;
    if (!cuda_ok(stage(kStageNormalRhs, ws->prec, a, st, ws), R)) return LSMGPU_ERR_CUDA;
    k_dt_finish<<<1, 256, 0, st>>>(ws->partials, nblk, cfl, tiny, ws->scal, 0.0);
    ++launch_counter();
    // stage 1: phi1 = phi + dt L (LSM3D_TVD_RK3_STAGE1)
    if (!cuda_ok(launch_rk(ws->prec, 1, ws->phi1, ws->gb, nullptr, ws->gb, phi,
                           ws->gb, ws->rhs, ws->gb, f, 0.0, ws->scal + kDt, st,
                           next_sr_seed(ws)),
                 R))
      return LSMGPU_ERR_CUDA;
    a.out = ws->phi2; a.phi_s = ws->phi1; a.phi_n = phi; a.rk_kind = 32;
    if (!cuda_ok(stage(kStageNormal, ws->prec, a, st, ws), R)) return LSMGPU_ERR_CUDA;
    a.out = phi; a.phi_s = ws->phi2; a.rk_kind = 33;
    if (!cuda_ok(stage(kStageNormal, ws->prec, a, st, ws), R)) return LSMGPU_ERR_CUDA;
    k_advance_t<<<1, 1, 0, st>>>(ws->scal);
    ++launch_counter();
    ws->steps++;
    if (reinit_interval > 0 && (step0 + s + 1) % reinit_interval == 0)
      if (!reinit_run(ws, phi, f, dx, cfl, reinit_iters, use_phi0_for_sgn, st, R))
        return lsmgpu_peek_last_error();
  }
  if (!cuda_ok(cudaGetLastError(), R)) return LSMGPU_ERR_CUDA;
  if (sync_mode() && !cuda_ok(cudaStreamSynchronize(st), R)) return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

// lsmgpu_normal_tvdrk3 on a level set and speed in host memory: phi and F are
// copied to the workspace's device buffers in kHostSlabs z-slabs while the
// first step's RHS/CFL pass works through the slabs already there, and the
// last step's final stage runs slab by slab, each slab copied back while the
// next is computed.  By default the call returns when phi is back in host
// memory.  With lsmgpu_workspace_set_host_async(ws, 1) it returns once its
// work is queued, and successive calls overlap: the speed goes to the next
// of nspeed device buffers while the previous call still computes, and each
// slab of phi is copied in as soon as the previous call's copy of that slab
// back to the host has landed (copies in, out and of the speed on three
// streams).
int lsmgpu_normal_tvdrk3_host(lsmgpu_workspace* ws, void* phi, const void* F,
                              const int fb[6], const double dx[3], double cfl, int nsteps,
                              int step0, int reinit_interval, int reinit_iters,
                              int use_phi0_for_sgn) {
  const char* R = "lsmgpu_normal_tvdrk3_host";
  FillBox f;
  if (!common_checks(ws, phi, fb, dx, R, &f)) return lsmgpu_peek_last_error();
  if (!F) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null speed");
    return LSMGPU_ERR_NULL_POINTER;
  }
  if (nsteps < 1) return LSMGPU_SUCCESS;
  cudaStream_t st = cur_stream();
  if (!ws->dphi) {
    if (!cuda_ok(cudaMalloc(&ws->dphi, ws->bytes), R) ||
        !cuda_ok(cudaMalloc(&ws->dF[0], ws->bytes), R) ||
        !cuda_ok(cudaStreamCreateWithFlags(&ws->copy_stream, cudaStreamNonBlocking), R) ||
        !cuda_ok(cudaStreamCreateWithFlags(&ws->copy_stream_out, cudaStreamNonBlocking), R) ||
        !cuda_ok(cudaStreamCreateWithFlags(&ws->copy_stream_F, cudaStreamNonBlocking), R) ||
        !cuda_ok(cudaEventCreateWithFlags(&ws->start_ev, cudaEventDisableTiming), R))
      return LSMGPU_ERR_CUDA;
    const size_t fit = ((size_t)1 << 30) / ws->bytes;
    ws->nspeed = fit < 2 ? 2 : fit > (size_t)kMaxSpeedBufs ? kMaxSpeedBufs : (int)fit;
    for (cudaEvent_t& e : ws->Fin_ev)
      if (!cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), R))
        return LSMGPU_ERR_CUDA;
    for (cudaEvent_t& e : ws->up_ev)
      if (!cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), R))
        return LSMGPU_ERR_CUDA;
    for (cudaEvent_t& e : ws->slab_ev)
      if (!cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), R))
        return LSMGPU_ERR_CUDA;
    for (cudaEvent_t& e : ws->out_ev)
      if (!cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), R))
        return LSMGPU_ERR_CUDA;
    for (cudaEvent_t& e : ws->F_ev)
      if (!cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), R))
        return LSMGPU_ERR_CUDA;
  }
  // queued calls take the speed buffers in turn and upload the speed on a
  // stream of its own (see the anchor below)
  const unsigned call = ws->host_calls;
  const int fbuf = ws->host_async ? (int)(call % (unsigned)ws->nspeed) : 0;
  if (!ws->dF[fbuf] && !cuda_ok(cudaMalloc(&ws->dF[fbuf], ws->bytes), R)) return LSMGPU_ERR_CUDA;
  void* dF = ws->dF[fbuf];
  cudaStream_t ci = ws->copy_stream, co = ws->copy_stream_out;
  cudaStream_t cf = ws->host_async ? ws->copy_stream_F : ci;
  const Box& gb = ws->gb;
  const size_t esz = (size_t)ws->prec;
  const size_t plane = (size_t)gb.sz() * esz;
  // fill-box slabs on stage-tile boundaries in z, and the ghost-box planes
  // each slab owns: [zb[s], zb[s+1]) with the ghost planes below the fill box
  // in the first and those above it in the last
  const int ntz = (f.n(2) + kStageTZ - 1) / kStageTZ;
  const int ns = ntz < kHostSlabs ? ntz : kHostSlabs;
  int zlo[kHostSlabs + 1];
  for (int q = 0; q <= ns; q++) zlo[q] = f.lo[2] + (int)((long)q * ntz / ns) * kStageTZ;
  zlo[ns] = f.hi[2] + 1;
  int zb[kHostSlabs + 1];
  for (int q = 0; q <= ns; q++) zb[q] = zlo[q];
  zb[0] = gb.lo[2];
  zb[ns] = gb.hi(2) + 1;
  auto slab_fb = [&](int q) {
    FillBox s = f;
    s.lo[2] = zlo[q];
    s.hi[2] = zlo[q + 1] - 1;
    return s;
  };
  auto copy = [&](void* dst, const void* src, int q, cudaMemcpyKind kind, cudaStream_t cs) {
    const size_t off = (size_t)(zb[q] - gb.lo[2]) * plane;
    return cudaMemcpyAsync((char*)dst + off, (const char*)src + off,
                           (size_t)(zb[q + 1] - zb[q]) * plane, kind, cs);
  };
  // host -> device.  After a waited-for call: behind all the work queued on
  // st.  Behind a queued call: the speed behind the last kernels that read
  // this buffer (nspeed calls back), each phi slab behind that call's copy
  // of the slab back to the host (which followed every kernel writing it).
  const bool pending = ws->host_pending != 0;
  if (!pending) {
    if (!cuda_ok(cudaEventRecord(ws->start_ev, st), R) ||
        !cuda_ok(cudaStreamWaitEvent(ci, ws->start_ev, 0), R) ||
        (cf != ci && !cuda_ok(cudaStreamWaitEvent(cf, ws->start_ev, 0), R)))
      return LSMGPU_ERR_CUDA;
  } else {
    // The speed of a queued call crosses the link after the previous call's
    // level set, so that it never delays a level-set upload (the next step
    // waits for it).  Behind a call that runs a reinitialization, the link
    // is idle while the level set is reinitialized: the speeds of the next
    // nspeed - 1 calls go right after that call's level set.
    const long long r = ws->last_reinit_call;
    const long long anchor = r >= 0 && (long long)call - r < ws->nspeed ? r : (long long)call - 1;
    if (!cuda_ok(cudaStreamWaitEvent(cf, ws->F_ev[fbuf], 0), R) ||
        (cf != ci && !cuda_ok(cudaStreamWaitEvent(cf, ws->up_ev[anchor % ws->nspeed], 0), R)))
      return LSMGPU_ERR_CUDA;
  }
  for (int q = 0; q < ns; q++)
    if (!cuda_ok(copy(dF, F, q, cudaMemcpyHostToDevice, cf), R)) return LSMGPU_ERR_CUDA;
  if (cf != ci && (!cuda_ok(cudaEventRecord(ws->Fin_ev[fbuf], cf), R) ||
                   !cuda_ok(cudaStreamWaitEvent(st, ws->Fin_ev[fbuf], 0), R)))
    return LSMGPU_ERR_CUDA;
  for (int q = 0; q < ns; q++) {
    if ((pending && !cuda_ok(cudaStreamWaitEvent(ci, ws->out_ev[q], 0), R)) ||
        !cuda_ok(copy(ws->dphi, phi, q, cudaMemcpyHostToDevice, ci), R) ||
        !cuda_ok(cudaEventRecord(ws->slab_ev[q], ci), R))
      return LSMGPU_ERR_CUDA;
  }
  if (!cuda_ok(cudaEventRecord(ws->up_ev[call % ws->nspeed], ci), R)) return LSMGPU_ERR_CUDA;
  const double tiny = ws->prec == 8 ? Consts<double>::tiny : (double)Consts<float>::tiny;
  const int nblk = stage_blocks(f);
  void* dphi = ws->dphi;
  bool copied_back = false;
  for (int s = 0; s < nsteps; s++) {
    StageArgs a = base_args(ws, f, dx);
    a.aux[0] = dF;
    a.rhs_out = ws->rhs;
    a.phi_s = dphi;
    if (s == 0) {
      // RHS/CFL pass of slab q once its planes and the 3 above have arrived
      int off = 0;
      for (int q = 0; q < ns; q++) {
        const int need = q + 1 < ns ? q + 1 : q;
        if (!cuda_ok(cudaStreamWaitEvent(st, ws->slab_ev[need], 0), R)) return LSMGPU_ERR_CUDA;
        StageArgs b = a;
        b.fb = slab_fb(q);
        b.partials = ws->partials + off;
        off += stage_blocks(b.fb);
        if (!cuda_ok(stage(kStageNormalRhs, ws->prec, b, st, ws), R)) return LSMGPU_ERR_CUDA;
      }
    } else {
      a.partials = ws->partials;
      if (!cuda_ok(stage(kStageNormalRhs, ws->prec, a, st, ws), R)) return LSMGPU_ERR_CUDA;
    }
    k_dt_finish<<<1, 256, 0, st>>>(ws->partials, nblk, cfl, tiny, ws->scal, 0.0);
    ++launch_counter();
    if (!cuda_ok(launch_rk(ws->prec, 1, ws->phi1, ws->gb, nullptr, ws->gb, dphi, ws->gb,
                           ws->rhs, ws->gb, f, 0.0, ws->scal + kDt, st, next_sr_seed(ws)),
                 R))
      return LSMGPU_ERR_CUDA;
    a.partials = ws->partials;
    a.out = ws->phi2; a.phi_s = ws->phi1; a.phi_n = dphi; a.rk_kind = 32;
    if (!cuda_ok(stage(kStageNormal, ws->prec, a, st, ws), R)) return LSMGPU_ERR_CUDA;
    a.out = dphi; a.phi_s = ws->phi2; a.rk_kind = 33;
    const bool reinit_now = reinit_interval > 0 && (step0 + s + 1) % reinit_interval == 0;
    if (reinit_now && reinit_iters > 0) ws->last_reinit_call = call;
    if (s == nsteps - 1 && !reinit_now) {
      // the final stage slab by slab, each slab's planes copied back at once
      for (int q = 0; q < ns; q++) {
        StageArgs b = a;
        b.fb = slab_fb(q);
        if (!cuda_ok(stage(kStageNormal, ws->prec, b, st, ws), R) ||
            !cuda_ok(cudaEventRecord(ws->slab_ev[kHostSlabs + q], st), R) ||
            !cuda_ok(cudaStreamWaitEvent(co, ws->slab_ev[kHostSlabs + q], 0), R) ||
            !cuda_ok(copy(phi, dphi, q, cudaMemcpyDeviceToHost, co), R) ||
            !cuda_ok(cudaEventRecord(ws->out_ev[q], co), R))
          return LSMGPU_ERR_CUDA;
      }
      copied_back = true;
    } else if (!cuda_ok(stage(kStageNormal, ws->prec, a, st, ws), R)) {
      return LSMGPU_ERR_CUDA;
    }
    k_advance_t<<<1, 1, 0, st>>>(ws->scal);
    ++launch_counter();
    ws->steps++;
    if (reinit_now && !reinit_run(ws, dphi, f, dx, cfl, reinit_iters, use_phi0_for_sgn, st, R))
      return lsmgpu_peek_last_error();
  }
  if (!cuda_ok(cudaEventRecord(ws->F_ev[fbuf], st), R)) return LSMGPU_ERR_CUDA;
  if (!copied_back) {
    if (!cuda_ok(cudaEventRecord(ws->slab_ev[kHostSlabs], st), R) ||
        !cuda_ok(cudaStreamWaitEvent(co, ws->slab_ev[kHostSlabs], 0), R))
      return LSMGPU_ERR_CUDA;
    for (int q = 0; q < ns; q++)
      if (!cuda_ok(copy(phi, dphi, q, cudaMemcpyDeviceToHost, co), R) ||
          !cuda_ok(cudaEventRecord(ws->out_ev[q], co), R))
        return LSMGPU_ERR_CUDA;
  }
  ws->host_calls++;
  if (!cuda_ok(cudaGetLastError(), R)) return LSMGPU_ERR_CUDA;
  if (ws->host_async) {
    ws->host_pending = 1;
    return LSMGPU_SUCCESS;
  }
  ws->host_pending = 0;
  if (!cuda_ok(cudaStreamSynchronize(co), R) || !cuda_ok(cudaStreamSynchronize(ci), R) ||
      !cuda_ok(cudaStreamSynchronize(st), R))
    return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

// reinitialization pseudo-steps alone (ReinitializationAlgorithm.cc:177-330)
int lsmgpu_reinit_tvdrk3(lsmgpu_workspace* ws, void* phi, const int fb[6],
                         const double dx[3], double cfl, int iters,
                         int use_phi0_for_sgn) {
  const char* R = "lsmgpu_reinit_tvdrk3";
  FillBox f;
  if (!common_checks(ws, phi, fb, dx, R, &f)) return lsmgpu_peek_last_error();
  cudaStream_t st = cur_stream();
  if (!reinit_run(ws, phi, f, dx, cfl, iters, use_phi0_for_sgn, st, R))
    return lsmgpu_peek_last_error();
  if (sync_mode() && !cuda_ok(cudaStreamSynchronize(st), R)) return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

}  // extern "C"
