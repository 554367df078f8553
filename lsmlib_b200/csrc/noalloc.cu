// noalloc.cu -- a normal-velocity RHS + CFL dt entry point that allocates
// nothing.
//
// Some callers cannot allocate device memory at the point where they call
// into the toolbox: code that runs under an allocator that forbids growth
// (a fixed memory pool reserved up front), a real-time loop whose latency
// budget cannot absorb cudaMalloc's device-wide synchronisation, or a host
// framework that owns all device memory and hands plug-ins only its own
// buffers.  lsmgpu_normal_rhs_dt_noalloc serves them: the caller passes the
// inputs and outputs, and the only scratch the kernel needs -- one partial
// CFL maximum per tile plus the dt result -- lives in the file-scope array
// below, which every GPU that loads this library keeps until the process
// exits.
#include <cstring>
#include <mutex>
#include <string>

#include "capi_common.h"
#include "launch.h"
#include "stage.cuh"
#include "stage_launch.h"

using namespace lsmgpu;

namespace {

// Scratch capacity: partial maxima of up to kNoAllocMaxTiles tiles of
// kStageTX x kStageTY x kStageTZ = 32 x 8 x 16 cells (8192 tiles cover
// 33.5 M cells, e.g. a 256^3 fill box needs 4096) plus one slot for dt.
constexpr int kNoAllocMaxTiles = 8192;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxTiles + 1];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device.  In host code g_noalloc_scratch names a host-side stand-in, so
// the kernels receive this address instead.
double* scratch_on_current_device(const char* R) {
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), R)) return nullptr;
  if (dev < 0 || dev >= kMaxDevices) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": device ordinal too large");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (!cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_scratch), R)) return nullptr;
    g_scratch_addr[dev] = (double*)p;
  }
  return g_scratch_addr[dev];
}

// dt = cfl / (max + tiny) from the first ``np`` partial maxima, with the
// reference's "if (h > m) m = h" comparison from m = -1
// (lsm_utilities3d.f.in:380-445).
__global__ void k_noalloc_dt(double* scratch, int np, double cfl, double tiny) {
  __shared__ double red[8];
  double m = -1.0;
  for (int t = threadIdx.x; t < np; t += blockDim.x) {
    const double v = scratch[t];
    m = (v > m) ? v : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_xor_sync(0xffffffffu, m, o);
    m = (v > m) ? v : m;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    m = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = (red[w] > m) ? red[w] : m;
    scratch[kNoAllocMaxTiles] = cfl / (m + tiny);
  }
}

}  // namespace

extern "C" int lsmgpu_normal_rhs_dt_noalloc(double* rhs, double* dt,
                                            const double* phi, const double* F,
                                            const int gb[6], const int fb[6],
                                            const double dx[3],
                                            double cfl_number) {
  const char* R = "lsmgpu_normal_rhs_dt_noalloc";
  clear_error();
  if (!rhs || !dt || !phi || !F || !gb || !fb || !dx) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  const Box g = box_from(&gb[0], &gb[1], &gb[2], &gb[3], &gb[4], &gb[5]);
  FillBox f;
  f.lo[0] = fb[0]; f.hi[0] = fb[1];
  f.lo[1] = fb[2]; f.hi[1] = fb[3];
  f.lo[2] = fb[4]; f.hi[2] = fb[5];
  if (f.n(0) < 1 || f.n(1) < 1 || f.n(2) < 1) {
    set_error(LSMGPU_ERR_INVALID_BOX, std::string(R) + ": empty fill box");
    return LSMGPU_ERR_INVALID_BOX;
  }
  if (!box_valid(g, "phi", R) || !covers(g, f, 3, "phi", R))
    return LSMGPU_ERR_INVALID_BOX;
  // the tile count in 64 bits: a box of more than 2^31 tiles must not wrap
  // around to a count that passes the check below
  const long tiles_l = (long)((f.n(0) + kStageTX - 1) / kStageTX) *
                       (long)((f.n(1) + kStageTY - 1) / kStageTY) *
                       (long)((f.n(2) + kStageTZ - 1) / kStageTZ);
  if (tiles_l > kNoAllocMaxTiles) {
    set_error(LSMGPU_ERR_INVALID_BOX,
              std::string(R) + ": fill box needs " + std::to_string(tiles_l) +
                  " tiles of " + std::to_string(kStageTX) + "x" + std::to_string(kStageTY) +
                  "x" + std::to_string(kStageTZ) + " cells; the static scratch holds " +
                  std::to_string(kNoAllocMaxTiles));
    return LSMGPU_ERR_INVALID_BOX;
  }
  const int tiles = (int)tiles_l;
  // host arrays would need staging buffers, i.e. an allocation
  if (!is_device_pointer(rhs) || !is_device_pointer(phi) || !is_device_pointer(F)) {
    set_error(LSMGPU_ERR_INVALID_VALUE,
              std::string(R) + ": rhs, phi and F must be device arrays");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  double* scratch = scratch_on_current_device(R);
  if (!scratch) return lsmgpu_peek_last_error();

  StageArgs a;
  memset(&a, 0, sizeof a);
  a.gb = g;
  a.fb = f;
  a.dom = f;
  a.bc_mask = 0u;  // ghost cells of phi are read as stored
  a.phi_s = phi;
  a.aux[0] = F;
  a.rhs_out = rhs;
  a.partials = scratch;
  for (int d = 0; d < 3; d++) a.inv[d] = 1.0 / dx[d];
  double m = dx[0] > dx[1] ? dx[0] : dx[1];
  m = m > dx[2] ? m : dx[2];
  a.dx_sq = m * m;
  cudaStream_t st = cur_stream();
  const cudaError_t e = fp_mode() == LSMGPU_FP_FAST
                            ? launch_stage_fast(kStageNormalRhs, 8, a, st)
                            : launch_stage_strict(kStageNormalRhs, 8, a, st);
  if (!cuda_ok(e, R)) return LSMGPU_ERR_CUDA;
  k_noalloc_dt<<<1, 256, 0, st>>>(scratch, tiles, cfl_number, Consts<double>::tiny);
  ++launch_counter();
  if (!cuda_ok(cudaGetLastError(), R)) return LSMGPU_ERR_CUDA;
  const cudaMemcpyKind kind = is_device_pointer(dt) ? cudaMemcpyDeviceToDevice
                                                    : cudaMemcpyDeviceToHost;
  if (!cuda_ok(cudaMemcpyAsync(dt, scratch + kNoAllocMaxTiles, sizeof(double),
                               kind, st),
               R))
    return LSMGPU_ERR_CUDA;
  if ((kind == cudaMemcpyDeviceToHost || sync_mode()) &&
      !cuda_ok(cudaStreamSynchronize(st), R))
    return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}
