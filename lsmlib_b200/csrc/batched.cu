// batched.cu -- many level-set grids of uneven sizes advanced together.
//
// The grids of a batch live in one packed device buffer (each grid's ghost
// box contiguous, 256-byte aligned).  A work-list holds one entry per tile
// (grid, tile x, tile y, tile z) of every grid.  Each TVD-RK3 stage is ONE
// persistent launch: every block takes the next tile from an atomic counter
// and runs the fused stage of stage.cuh on it, until the list is exhausted;
// blocks never wait for one another.  A whole step (three stages and the
// counter resets) is captured once in a CUDA graph and replayed.
//
// Each grid has its own constant velocity and its own CFL dt
//   dt = cfl / (|u|/dx + |v|/dy + |w|/dz + tiny)
// -- the value LSM3D_COMPUTE_STABLE_ADVECTION_DT returns for a constant field
// (lsm_utilities3d.f.in:299-322), kept in FP64.
//
// The tile shape (TX x TY cells, TZ planes) is chosen per batch by timing the
// candidates on the batch itself (lsmgpu_batch_autotune); the choice is
// cached per (precision, size class).
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "capi_common.h"
#include "launch.h"
#include "stage.cuh"

using namespace lsmgpu;

namespace {

struct GridMeta {
  long offset;     // element offset of the grid's ghost box
  Box gb;
  FillBox fb;
  double inv[3];
  double dx_sq;
  double dt;
  double vel[3];
};

// tile shapes the autotuner chooses from, each with three halo-staging
// schedules: 0 and 1 are stage_tile's STAGING (one cell per thread; x/y
// stencils through a shared plane with its side strips, or straight from
// global memory), 2 is stage_tile_pairs_up (two cells per thread, shared
// plane, one barrier per plane; needs the ghost cells stored).
// Configuration c is shape c % kNumShapes with schedule c / kNumShapes.
struct TileShape { int tx, ty, tz; };
constexpr TileShape kShapes[] = {{32, 8, 16}, {32, 8, 32}, {32, 8, 64}, {16, 8, 16},
                                 {16, 8, 32}};
constexpr int kNumShapes = 5;
constexpr int kNumStagings = 3;
constexpr int kNumConfigs = kNumShapes * kNumStagings;
constexpr int kPairStaging = 2;

// threads per block of a schedule, and the blocks per SM its register
// budget allows (one cell per thread: LSMGPU_BATCH_WARPS warps per SM; two
// cells per thread: 16 warps, the budget of the single-grid pair kernels)
#define BATCH_THREADS(TX, TY, SG) ((SG) == kPairStaging ? (TX) / 2 * (TY) : (TX) * (TY))
#define BATCH_MIN_BLOCKS(TX, TY, SG) \
  ((SG) == kPairStaging ? 512 / ((TX) / 2 * (TY)) : LSMGPU_BATCH_WARPS * 32 / ((TX) * (TY)))

// seed of the stochastic rounding of one stage: the step number kept on the
// device (bumped at the end of every step, so that graph replays differ)
// and the stage
template <typename T>
__device__ __forceinline__ unsigned batch_sr_seed(int policy, const unsigned* sr_step,
                                                  int rk_kind) {
  if (sizeof(T) != 4 || !(policy & kStochRound) || !sr_step) return 0u;
  return sr_hash(*sr_step * 64u + (unsigned)rk_kind) | 1u;
}

__global__ void k_bump(unsigned* c) { *c += 1u; }

// register budget: 24 warps per SM, as the single-grid stage kernels (the
// earlier budget of 2 blocks let the compiler take 190 registers and left
// the SMs at 8 warps: ncu, 12 % warps active, 45 % issue)
#ifndef LSMGPU_BATCH_WARPS
#define LSMGPU_BATCH_WARPS 24
#endif

// one tile of the batch with a schedule's stage routine
template <typename T, int TX, int TY, int TZ, int STAGING>
__device__ __forceinline__ void batch_tile(const StageParams<T>& p, int bx, int by, int bz,
                                           int policy) {
  if constexpr (STAGING == kPairStaging) {
    __shared__ __align__(16) T tile[2][TY + 6][TX + 8];
    if (sizeof(T) == 4 && (policy & kFp64Kinks))
      stage_tile_pairs_up<T, kStageAdvectConst, sizeof(T) == 4, TX, TY, TZ>(p, bx, by, bz, tile);
    else
      stage_tile_pairs_up<T, kStageAdvectConst, false, TX, TY, TZ>(p, bx, by, bz, tile);
  } else {
    __shared__ T tile[2][TY + 6][TX + 6];
    stage_tile<T, kStageAdvectConst, true, TX, TY, TZ, STAGING>(p, bx, by, bz, tile);
  }
}

template <typename T, int TX, int TY, int TZ, int STAGING>
__global__ void __launch_bounds__(BATCH_THREADS(TX, TY, STAGING),
                                  BATCH_MIN_BLOCKS(TX, TY, STAGING))
k_batched_stage(const GridMeta* __restrict__ grids, const int4* __restrict__ items,
                int nitems, unsigned* counter, T* out, const T* phi_s,
                const T* phi_n, int rk_kind, int policy, const unsigned* sr_step,
                unsigned bc_mask) {
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0 && threadIdx.y == 0) s_item = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int t = s_item;
    // every thread has read s_item and finished the previous tile
    __syncthreads();
    if (t >= nitems) break;
    const int4 it = items[t];
    const GridMeta& g = grids[it.x];
    StageParams<T> p;
    p.out = out + g.offset;
    p.phi_s = phi_s + g.offset;
    p.phi_n = phi_n + g.offset;
    p.aux0 = p.aux1 = p.aux2 = nullptr;
    p.rhs_out = nullptr;
    p.partials = nullptr;
    p.gb = g.gb;
    p.fb = g.fb;
    p.dom = g.fb;
    p.bc_mask = bc_mask;
    for (int d = 0; d < 3; d++) {
      p.inv[d] = (T)g.inv[d];
      p.fk[d] = face_const<T>(p.inv[d]);
      p.vel_const[d] = (T)g.vel[d];
    }
    p.dx_sq = (T)g.dx_sq;
    p.dt_dev = nullptr;
    p.dt = g.dt;
    p.rk_kind = rk_kind;
    p.use_phi0 = 0;
    p.fp64_policy = policy & kFp64Kinks;
    p.sr_seed = batch_sr_seed<T>(policy, sr_step, rk_kind);
    batch_tile<T, TX, TY, TZ, STAGING>(p, it.y, it.z, it.w, policy);
  }
}

// The face ghost cells of every grid of a packed buffer, written as stored
// values before a stage (the kinds of fetch_bc, through face_ghost_value), so
// that the stage reads them from memory: with grids of 32-128 cells per axis
// nearly every tile touches a face, and generating them on the fly put the
// boundary branch in nearly every load.  Item (g, k >= 0): the x and y ghost
// rows of plane k of grid g; item (g, -1 - p): z ghost plane p (side * 3 +
// layer).  Every value depends on domain cells only.
template <typename T>
__global__ void __launch_bounds__(128)
k_batched_ghosts(const GridMeta* __restrict__ grids, const int2* __restrict__ items,
                 int nitems, T* buf, unsigned m) {
  for (int q = blockIdx.x; q < nitems; q += gridDim.x) {
    const int2 it = items[q];
    const GridMeta& g = grids[it.x];
    const FillBox dom = g.fb;
    const Grid3<T> gr = make_grid(buf + g.offset, g.gb);
    const int nx = dom.n(0), ny = dom.n(1);
    auto has = [&](int face) {
      return ((m >> face) | (m >> (8 + face)) | (m >> (16 + face))) & 1u;
    };
    if (it.y >= 0) {
      const int k = dom.lo[2] + it.y;
      ghost_items<4, T>(threadIdx.x, 6 * ny, blockDim.x, [&](int r, T& v) -> T* {
        const int j = dom.lo[1] + r / 6, face = (r % 6) / 3, dist = r % 3 + 1;
        if (!has(face)) return nullptr;
        const int i = face ? dom.hi[0] + dist : dom.lo[0] - dist;
        T* const cell = gr.ptr(i, j, k);
        v = face_ghost_value(gr, dom, m, face, dist, cell);
        return cell;
      });
      ghost_items<4, T>(threadIdx.x, 6 * nx, blockDim.x, [&](int r, T& v) -> T* {
        const int i = dom.lo[0] + r % nx, face = 2 + (r / nx) / 3, dist = (r / nx) % 3 + 1;
        if (!has(face)) return nullptr;
        const int j = face == 3 ? dom.hi[1] + dist : dom.lo[1] - dist;
        T* const cell = gr.ptr(i, j, k);
        v = face_ghost_value(gr, dom, m, face, dist, cell);
        return cell;
      });
    } else {
      const int zp = -1 - it.y, face = 4 + zp / 3, dist = zp % 3 + 1;
      if (!has(face)) continue;
      const int k = face == 5 ? dom.hi[2] + dist : dom.lo[2] - dist;
      ghost_items<4, T>(threadIdx.x, nx * ny, blockDim.x, [&](int r, T& v) -> T* {
        const int i = dom.lo[0] + r % nx, j = dom.lo[1] + r / nx;
        T* const cell = gr.ptr(i, j, k);
        v = face_ghost_value(gr, dom, m, face, dist, cell);
        return cell;
      });
    }
  }
}

// the plain alternative: one launch per grid per stage
template <typename T, int TX, int TY, int TZ, int STAGING>
__global__ void __launch_bounds__(BATCH_THREADS(TX, TY, STAGING),
                                  BATCH_MIN_BLOCKS(TX, TY, STAGING))
k_grid_stage(const GridMeta* __restrict__ grids, int gi, T* out, const T* phi_s,
             const T* phi_n, int rk_kind, int policy, const unsigned* sr_step,
             unsigned bc_mask) {
  const GridMeta& g = grids[gi];
  StageParams<T> p;
  p.out = out + g.offset;
  p.phi_s = phi_s + g.offset;
  p.phi_n = phi_n + g.offset;
  p.aux0 = p.aux1 = p.aux2 = nullptr;
  p.rhs_out = nullptr;
  p.partials = nullptr;
  p.gb = g.gb;
  p.fb = g.fb;
  p.dom = g.fb;
  p.bc_mask = bc_mask;
  for (int d = 0; d < 3; d++) {
    p.inv[d] = (T)g.inv[d];
      p.fk[d] = face_const<T>(p.inv[d]);
    p.vel_const[d] = (T)g.vel[d];
  }
  p.dx_sq = (T)g.dx_sq;
  p.dt_dev = nullptr;
  p.dt = g.dt;
  p.rk_kind = rk_kind;
  p.use_phi0 = 0;
  p.fp64_policy = policy & kFp64Kinks;
  p.sr_seed = batch_sr_seed<T>(policy, sr_step, rk_kind);
  batch_tile<T, TX, TY, TZ, STAGING>(p, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, policy);
}

std::mutex g_tune_mutex;
std::map<std::pair<int, int>, int> g_tune_cache;   // (precision, size class) -> shape

}  // namespace

struct lsmgpu_batch {
  int ngrids = 0;
  int prec = 8;
  std::vector<GridMeta> meta;       // host copy
  GridMeta* d_meta = nullptr;
  long total = 0;                   // elements in each packed buffer
  long cells = 0;                   // interior cells of all grids
  void* phi = nullptr;
  void* phi1 = nullptr;
  void* phi2 = nullptr;
  int4* d_items[kNumShapes] = {nullptr};
  int nitems[kNumShapes] = {0};
  // ghost-fill items (see k_batched_ghosts); ghosts_stored: every grid has
  // at least 3 cells per axis, so the ghosts are written before each stage
  int2* d_ghost_items = nullptr;
  int n_ghost_items = 0;
  bool ghosts_stored = false;
  unsigned* d_counter = nullptr;    // three tile counters (one per stage), step
  int shape = 1;
  int policy = kStochRound;         // FP32: kFp64Kinks | kStochRound
  unsigned bc_mask = kBcLinear;
  int blocks_per_sm = 2;
  int resident[kNumConfigs] = {0};   // blocks per SM of each configuration's kernel
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_shape = -1;
};

namespace {

int size_class(const lsmgpu_batch* b) {
  // mean interior edge length bucketed by powers of two
  const double mean = b->ngrids ? (double)b->cells / b->ngrids : 0.0;
  int c = 0;
  for (double e = std::cbrt(mean); e >= 2.0; e /= 2.0) c++;
  return c;
}

template <typename T>
cudaError_t launch_shape(lsmgpu_batch* b, int shape, bool batched, int rk_kind,
                         T* out, const T* in, const T* base, unsigned* counter,
                         cudaStream_t st) {
  // persistent grid: every SM filled with as many blocks of the
  // configuration as fit.  The two-cells-per-thread schedule reads the ghost
  // cells as stored; without them (a grid with fewer than 3 cells along an
  // axis) its shape runs with schedule 0.
  int cfg = shape;
  if (cfg / kNumShapes == kPairStaging && !b->ghosts_stored) cfg %= kNumShapes;
  shape = cfg % kNumShapes;
  const int sg = cfg / kNumShapes;
  const int threads = sg == kPairStaging ? kShapes[shape].tx / 2 * kShapes[shape].ty
                                         : kShapes[shape].tx * kShapes[shape].ty;
#define BATCH_CONFIGS(X)                                                           \
  X(0, 32, 8, 16, 0) X(1, 32, 8, 32, 0) X(2, 32, 8, 64, 0) X(3, 16, 8, 16, 0)      \
  X(4, 16, 8, 32, 0) X(5, 32, 8, 16, 1) X(6, 32, 8, 32, 1) X(7, 32, 8, 64, 1)      \
  X(8, 16, 8, 16, 1) X(9, 16, 8, 32, 1) X(10, 32, 8, 16, 2) X(11, 32, 8, 32, 2)    \
  X(12, 32, 8, 64, 2) X(13, 16, 8, 16, 2) X(14, 16, 8, 32, 2)
  if (b->resident[cfg] == 0) {
    const void* fn = nullptr;
#define BATCH_FN(I, TX, TY, TZ, SG) \
  case I: fn = (const void*)k_batched_stage<T, TX, TY, TZ, SG>; break;
    switch (cfg) {
      BATCH_CONFIGS(BATCH_FN)
      default: return cudaErrorInvalidValue;
    }
#undef BATCH_FN
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, 0) != cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = b->blocks_per_sm;
    }
    b->resident[cfg] = nb;
  }
  const int grid = b->num_sms * b->resident[cfg];
  // with stored ghosts the stage reads every ghost cell from memory
  unsigned bcm = b->bc_mask;
  if (b->ghosts_stored) {
    const int gblocks = std::min(b->n_ghost_items, b->num_sms * 8);
    k_batched_ghosts<T><<<gblocks, 128, 0, st>>>(b->d_meta, b->d_ghost_items,
                                                b->n_ghost_items, (T*)in, b->bc_mask);
    ++launch_counter();
    bcm = 0u;
  }
#define BATCH_CASE(I, TX, TY, TZ, SG)                                              \
  case I:                                                                          \
    if (batched) {                                                                 \
      k_batched_stage<T, TX, TY, TZ, SG><<<grid, dim3(BATCH_THREADS(TX, TY, SG) / (TY), TY), 0, st>>>( \
          b->d_meta, b->d_items[I % kNumShapes], b->nitems[I % kNumShapes], counter, \
          out, in, base, rk_kind, b->policy, b->d_counter + 3, bcm);               \
    } else {                                                                       \
      for (int gi = 0; gi < b->ngrids; gi++) {                                     \
        const FillBox& f = b->meta[gi].fb;                                         \
        dim3 g((f.n(0) + TX - 1) / TX, (f.n(1) + TY - 1) / TY, (f.n(2) + TZ - 1) / TZ); \
        k_grid_stage<T, TX, TY, TZ, SG><<<g, dim3(BATCH_THREADS(TX, TY, SG) / (TY), TY), 0, st>>>( \
            b->d_meta, gi, out, in, base, rk_kind, b->policy, b->d_counter + 3,    \
            bcm);                                                                  \
      }                                                                            \
    }                                                                              \
    break;
  switch (cfg) {
    BATCH_CONFIGS(BATCH_CASE)
    default: return cudaErrorInvalidValue;
  }
#undef BATCH_CASE
#undef BATCH_CONFIGS
  launch_counter() += batched ? 1 : b->ngrids;
  return cudaGetLastError();
}

// one TVD-RK3 step of every grid (phi in place)
cudaError_t step(lsmgpu_batch* b, int shape, bool batched, cudaStream_t st) {
  cudaError_t e;
  for (int s = 0; s < 3; s++)
    if ((e = cudaMemsetAsync(b->d_counter + s, 0, sizeof(unsigned), st)) != cudaSuccess)
      return e;
  if (b->prec == 8) {
    double *phi = (double*)b->phi, *p1 = (double*)b->phi1, *p2 = (double*)b->phi2;
    if ((e = launch_shape<double>(b, shape, batched, 1, p1, phi, phi, b->d_counter, st))) return e;
    if ((e = launch_shape<double>(b, shape, batched, 32, p2, p1, phi, b->d_counter + 1, st))) return e;
    return launch_shape<double>(b, shape, batched, 33, phi, p2, phi, b->d_counter + 2, st);
  }
  float *phi = (float*)b->phi, *p1 = (float*)b->phi1, *p2 = (float*)b->phi2;
  if ((e = launch_shape<float>(b, shape, batched, 1, p1, phi, phi, b->d_counter, st))) return e;
  if ((e = launch_shape<float>(b, shape, batched, 32, p2, p1, phi, b->d_counter + 1, st))) return e;
  if ((e = launch_shape<float>(b, shape, batched, 33, phi, p2, phi, b->d_counter + 2, st))) return e;
  if (b->policy & kStochRound) {
    k_bump<<<1, 1, 0, st>>>(b->d_counter + 3);
    ++launch_counter();
    return cudaGetLastError();
  }
  return cudaSuccess;
}

bool batch_ok(lsmgpu_batch* b, const char* R) {
  if (!b) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null batch");
    return false;
  }
  return true;
}

void drop_graph(lsmgpu_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_shape = -1;
}

}  // namespace

extern "C" {

// ngrids grids with interior sizes n[3*g..3*g+2] (cells 0..n-1 per axis, 3
// ghost cells per side) and spacings dx[3*g..3*g+2].
int lsmgpu_batch_create(lsmgpu_batch** out, int ngrids, const int* n,
                        const double* dx, int precision) {
  const char* R = "lsmgpu_batch_create";
  clear_error();
  if (!out || !n || !dx) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null argument");
    return LSMGPU_ERR_NULL_POINTER;
  }
  *out = nullptr;
  if (ngrids < 1 || (precision != 8 && precision != 4)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, std::string(R) + ": bad count/precision");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  lsmgpu_batch* b = new lsmgpu_batch();
  b->ngrids = ngrids;
  b->prec = precision;
  b->policy = kStochRound;
  long off = 0;
  const long align = 256 / precision;
  for (int g = 0; g < ngrids; g++) {
    GridMeta m;
    memset(&m, 0, sizeof m);
    for (int d = 0; d < 3; d++) {
      if (n[3 * g + d] < 2 || !(dx[3 * g + d] > 0)) {
        set_error(LSMGPU_ERR_INVALID_BOX, std::string(R) + ": grid needs >= 2 cells "
                                                         "per axis and dx > 0");
        delete b;
        return LSMGPU_ERR_INVALID_BOX;
      }
      m.gb.lo[d] = -3;
      m.gb.n[d] = n[3 * g + d] + 6;
      m.fb.lo[d] = 0;
      m.fb.hi[d] = n[3 * g + d] - 1;
      m.inv[d] = 1.0 / dx[3 * g + d];
    }
    double mx = dx[3 * g] > dx[3 * g + 1] ? dx[3 * g] : dx[3 * g + 1];
    mx = mx > dx[3 * g + 2] ? mx : dx[3 * g + 2];
    m.dx_sq = mx * mx;
    m.offset = off;
    off += (m.gb.count() + align - 1) / align * align;
    b->cells += m.fb.count();
    b->meta.push_back(m);
  }
  b->total = off;
  const size_t bytes = (size_t)off * precision;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, dev);
  bool ok = cudaMalloc(&b->phi, bytes) == cudaSuccess &&
            cudaMalloc(&b->phi1, bytes) == cudaSuccess &&
            cudaMalloc(&b->phi2, bytes) == cudaSuccess &&
            cudaMalloc((void**)&b->d_meta, sizeof(GridMeta) * ngrids) == cudaSuccess &&
            cudaMalloc((void**)&b->d_counter, sizeof(unsigned) * 4) == cudaSuccess &&
            cudaMemset(b->d_counter, 0, sizeof(unsigned) * 4) == cudaSuccess;
  // work-lists for every candidate tile shape, largest tiles first
  for (int s = 0; ok && s < kNumShapes; s++) {
    std::vector<int4> items;
    std::vector<long> cost;
    for (int g = 0; g < ngrids; g++) {
      const FillBox& f = b->meta[g].fb;
      const int gx = (f.n(0) + kShapes[s].tx - 1) / kShapes[s].tx;
      const int gy = (f.n(1) + kShapes[s].ty - 1) / kShapes[s].ty;
      const int gz = (f.n(2) + kShapes[s].tz - 1) / kShapes[s].tz;
      for (int z = 0; z < gz; z++)
        for (int y = 0; y < gy; y++)
          for (int x = 0; x < gx; x++) {
            items.push_back(make_int4(g, x, y, z));
            const long cx = std::min(kShapes[s].tx, f.n(0) - x * kShapes[s].tx);
            const long cy = std::min(kShapes[s].ty, f.n(1) - y * kShapes[s].ty);
            const long cz = std::min(kShapes[s].tz, f.n(2) - z * kShapes[s].tz);
            cost.push_back(cx * cy * cz);
          }
    }
    std::vector<int> order(items.size());
    for (size_t q = 0; q < order.size(); q++) order[q] = (int)q;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return cost[a] > cost[c]; });
    std::vector<int4> sorted(items.size());
    for (size_t q = 0; q < order.size(); q++) sorted[q] = items[order[q]];
    b->nitems[s] = (int)sorted.size();
    ok = cudaMalloc((void**)&b->d_items[s], sizeof(int4) * sorted.size()) == cudaSuccess &&
         cudaMemcpy(b->d_items[s], sorted.data(), sizeof(int4) * sorted.size(),
                    cudaMemcpyHostToDevice) == cudaSuccess;
  }
  // ghost-fill items: every plane of every grid, and its 6 z ghost planes
  b->ghosts_stored = true;
  for (int g = 0; g < ngrids; g++)
    for (int d = 0; d < 3; d++)
      if (b->meta[g].fb.n(d) < 3) b->ghosts_stored = false;
  if (ok && b->ghosts_stored) {
    std::vector<int2> gi;
    for (int g = 0; g < ngrids; g++) {
      for (int k = 0; k < b->meta[g].fb.n(2); k++) gi.push_back(make_int2(g, k));
      for (int zp = 0; zp < 6; zp++) gi.push_back(make_int2(g, -1 - zp));
    }
    b->n_ghost_items = (int)gi.size();
    ok = cudaMalloc((void**)&b->d_ghost_items, sizeof(int2) * gi.size()) == cudaSuccess &&
         cudaMemcpy(b->d_ghost_items, gi.data(), sizeof(int2) * gi.size(),
                    cudaMemcpyHostToDevice) == cudaSuccess;
  }
  ok = ok && cudaMemset(b->phi, 0, bytes) == cudaSuccess &&
       cudaMemset(b->phi1, 0, bytes) == cudaSuccess &&
       cudaMemset(b->phi2, 0, bytes) == cudaSuccess &&
       cudaMemcpy(b->d_meta, b->meta.data(), sizeof(GridMeta) * ngrids,
                  cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    set_error(LSMGPU_ERR_ALLOC, std::string(R) + ": device allocation failed");
    lsmgpu_batch_destroy(b);
    return LSMGPU_ERR_ALLOC;
  }
  *out = b;
  return LSMGPU_SUCCESS;
}

int lsmgpu_batch_destroy(lsmgpu_batch* b) {
  if (!b) return LSMGPU_SUCCESS;
  drop_graph(b);
  void* ps[] = {b->phi, b->phi1, b->phi2, b->d_meta, b->d_counter, b->d_ghost_items};
  for (void* p : ps)
    if (p) cudaFree(p);
  for (int s = 0; s < kNumShapes; s++)
    if (b->d_items[s]) cudaFree(b->d_items[s]);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return LSMGPU_SUCCESS;
}

// element offset of grid g in the packed buffer and its ghost box
int lsmgpu_batch_grid(lsmgpu_batch* b, int g, long long* offset, int gb[6]) {
  if (!batch_ok(b, "lsmgpu_batch_grid")) return LSMGPU_ERR_NULL_POINTER;
  if (g < 0 || g >= b->ngrids) {
    set_error(LSMGPU_ERR_INVALID_VALUE, "lsmgpu_batch_grid: grid index out of range");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  const GridMeta& m = b->meta[g];
  if (offset) *offset = m.offset;
  if (gb)
    for (int d = 0; d < 3; d++) {
      gb[2 * d] = m.gb.lo[d];
      gb[2 * d + 1] = m.gb.hi(d);
    }
  return LSMGPU_SUCCESS;
}

// copy the whole packed phi buffer from/to the host (grid g at its offset)
int lsmgpu_batch_upload(lsmgpu_batch* b, const void* host) {
  if (!batch_ok(b, "lsmgpu_batch_upload")) return LSMGPU_ERR_NULL_POINTER;
  return cuda_ok(cudaMemcpy(b->phi, host, (size_t)b->total * b->prec,
                            cudaMemcpyHostToDevice),
                 "lsmgpu_batch_upload")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}
int lsmgpu_batch_download(lsmgpu_batch* b, void* host) {
  if (!batch_ok(b, "lsmgpu_batch_download")) return LSMGPU_ERR_NULL_POINTER;
  if (!cuda_ok(cudaStreamSynchronize(b->stream), "lsmgpu_batch_download"))
    return LSMGPU_ERR_CUDA;
  return cuda_ok(cudaMemcpy(host, b->phi, (size_t)b->total * b->prec,
                            cudaMemcpyDeviceToHost),
                 "lsmgpu_batch_download")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}
long long lsmgpu_batch_total_elements(lsmgpu_batch* b) { return b ? b->total : 0; }
long long lsmgpu_batch_cells(lsmgpu_batch* b) { return b ? b->cells : 0; }

// constant velocity of every grid (3 per grid) and the CFL number: sets each
// grid's dt = cfl / (|u|/dx + |v|/dy + |w|/dz + tiny)
int lsmgpu_batch_set_velocity(lsmgpu_batch* b, const double* vel, double cfl) {
  const char* R = "lsmgpu_batch_set_velocity";
  if (!batch_ok(b, R)) return LSMGPU_ERR_NULL_POINTER;
  if (!vel) {
    set_error(LSMGPU_ERR_NULL_POINTER, std::string(R) + ": null velocity");
    return LSMGPU_ERR_NULL_POINTER;
  }
  const double tiny = b->prec == 8 ? Consts<double>::tiny : (double)Consts<float>::tiny;
  for (int g = 0; g < b->ngrids; g++) {
    GridMeta& m = b->meta[g];
    for (int d = 0; d < 3; d++) m.vel[d] = vel[3 * g + d];
    const double u = fabs(m.vel[0]) * m.inv[0] + fabs(m.vel[1]) * m.inv[1] +
                     fabs(m.vel[2]) * m.inv[2];
    m.dt = cfl / (u + tiny);
  }
  drop_graph(b);
  return cuda_ok(cudaMemcpy(b->d_meta, b->meta.data(), sizeof(GridMeta) * b->ngrids,
                            cudaMemcpyHostToDevice),
                 R)
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}

int lsmgpu_batch_get_dt(lsmgpu_batch* b, double* dt) {
  if (!batch_ok(b, "lsmgpu_batch_get_dt") || !dt) return LSMGPU_ERR_NULL_POINTER;
  for (int g = 0; g < b->ngrids; g++) dt[g] = b->meta[g].dt;
  return LSMGPU_SUCCESS;
}

// configuration: tile shape (shape % 5 of the list above) and halo-staging
// schedule (shape / 5: 0 shared plane, 1 direct loads, 2 two cells per
// thread)
int lsmgpu_batch_set_tile(lsmgpu_batch* b, int shape) {
  if (!batch_ok(b, "lsmgpu_batch_set_tile")) return LSMGPU_ERR_NULL_POINTER;
  if (shape < 0 || shape >= kNumConfigs) {
    set_error(LSMGPU_ERR_INVALID_VALUE, "lsmgpu_batch_set_tile: unknown shape");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  if (shape != b->shape) drop_graph(b);
  b->shape = shape;
  return LSMGPU_SUCCESS;
}
int lsmgpu_batch_get_tile(lsmgpu_batch* b, int* shape, int tile[3]) {
  if (!batch_ok(b, "lsmgpu_batch_get_tile")) return LSMGPU_ERR_NULL_POINTER;
  if (shape) *shape = b->shape;
  if (tile) {
    tile[0] = kShapes[b->shape % kNumShapes].tx;
    tile[1] = kShapes[b->shape % kNumShapes].ty;
    tile[2] = kShapes[b->shape % kNumShapes].tz;
  }
  return LSMGPU_SUCCESS;
}
// boundary kind of every grid: 0 linear extrapolation, 1 copy (homogeneous
// Neumann), 2 periodic
int lsmgpu_batch_set_bc(lsmgpu_batch* b, int kind) {
  if (!batch_ok(b, "lsmgpu_batch_set_bc")) return LSMGPU_ERR_NULL_POINTER;
  if (kind < 0 || kind > 2) {
    set_error(LSMGPU_ERR_INVALID_VALUE, "lsmgpu_batch_set_bc: kind is 0, 1 or 2");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  b->bc_mask = kind == 0 ? kBcLinear : (kind == 1 ? kBcCopy : kBcPeriodic);
  drop_graph(b);
  return LSMGPU_SUCCESS;
}

// FP32 batches: recompute kink stencils in FP64 (0 off, 1 on)
int lsmgpu_batch_set_fp64_kinks(lsmgpu_batch* b, int on) {
  if (!batch_ok(b, "lsmgpu_batch_set_fp64_kinks")) return LSMGPU_ERR_NULL_POINTER;
  b->policy = (b->policy & ~kFp64Kinks) | (on ? kFp64Kinks : 0);
  drop_graph(b);
  return LSMGPU_SUCCESS;
}

// FP32 batches: bit 0 kink stencils in FP64, bit 2 stochastic rounding of the
// stage outputs (bit 1, the reinitialization sign, has no stage here)
int lsmgpu_batch_set_fp64_policy(lsmgpu_batch* b, int policy) {
  if (!batch_ok(b, "lsmgpu_batch_set_fp64_policy")) return LSMGPU_ERR_NULL_POINTER;
  if (policy & ~(kFp64Kinks | kFp64Sign | kStochRound)) {
    set_error(LSMGPU_ERR_INVALID_VALUE, "lsmgpu_batch_set_fp64_policy: unknown bits");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  b->policy = policy;
  drop_graph(b);
  return LSMGPU_SUCCESS;
}

// Time one step per tile shape (on a scratch copy of phi, so the batch state
// is unchanged) and keep the fastest; the choice is cached per (precision,
// size class).  ms_out[10] receives the timings of the ten configurations
// (tile shape x halo-staging schedule) when non-null.
int lsmgpu_batch_autotune(lsmgpu_batch* b, float* ms_out) {
  const char* R = "lsmgpu_batch_autotune";
  if (!batch_ok(b, R)) return LSMGPU_ERR_NULL_POINTER;
  const std::pair<int, int> key(b->prec, size_class(b));
  if (!ms_out) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) return lsmgpu_batch_set_tile(b, it->second);
  }
  const size_t bytes = (size_t)b->total * b->prec;
  void* save = nullptr;
  if (!cuda_ok(cudaMalloc(&save, bytes), R)) return LSMGPU_ERR_ALLOC;
  cudaMemcpyAsync(save, b->phi, bytes, cudaMemcpyDeviceToDevice, b->stream);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = b->shape;
  float best_ms = 1e30f;
  for (int s = 0; s < kNumConfigs; s++) {
    float ms = 0.f;
    bool ok = step(b, s, true, b->stream) == cudaSuccess;  // warm-up
    ok = ok && cudaEventRecord(e0, b->stream) == cudaSuccess;
    for (int r = 0; ok && r < 3; r++) ok = step(b, s, true, b->stream) == cudaSuccess;
    ok = ok && cudaEventRecord(e1, b->stream) == cudaSuccess &&
         cudaEventSynchronize(e1) == cudaSuccess &&
         cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
    if (!ok) {
      cuda_ok(cudaGetLastError(), R);
      break;
    }
    if (ms_out) ms_out[s] = ms / 3;
    if (ms < best_ms) {
      best_ms = ms;
      best = s;
    }
  }
  cudaMemcpyAsync(b->phi, save, bytes, cudaMemcpyDeviceToDevice, b->stream);
  cudaStreamSynchronize(b->stream);
  cudaFree(save);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tune_cache[key] = best;
  }
  return lsmgpu_batch_set_tile(b, best);
}

// nsteps TVD-RK3 steps of every grid.  mode 0: persistent work-list launches
// replayed from a CUDA graph; 1: the same launches without a graph; 2: one
// launch per grid per stage (the plain path, for comparison).  Runs on the
// batch's own stream; waits for completion when ``sync``.
int lsmgpu_batch_advect_tvdrk3(lsmgpu_batch* b, int nsteps, int mode, int sync) {
  const char* R = "lsmgpu_batch_advect_tvdrk3";
  clear_error();
  if (!batch_ok(b, R)) return LSMGPU_ERR_NULL_POINTER;
  if (mode == 0) {
    if (!b->exec || b->graph_shape != b->shape) {
      drop_graph(b);
      if (!cuda_ok(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), R))
        return LSMGPU_ERR_CUDA;
      const cudaError_t e = step(b, b->shape, true, b->stream);
      cudaGraph_t g = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
      if (!cuda_ok(e, R) || !cuda_ok(e2, R)) {
        if (g) cudaGraphDestroy(g);
        return LSMGPU_ERR_CUDA;
      }
      b->graph = g;
      if (!cuda_ok(cudaGraphInstantiate(&b->exec, b->graph, 0), R)) {
        drop_graph(b);
        return LSMGPU_ERR_CUDA;
      }
      b->graph_shape = b->shape;
    }
    for (int s = 0; s < nsteps; s++) {
      if (!cuda_ok(cudaGraphLaunch(b->exec, b->stream), R)) return LSMGPU_ERR_CUDA;
      launch_counter() += 3;
    }
  } else {
    for (int s = 0; s < nsteps; s++)
      if (!cuda_ok(step(b, b->shape, mode == 1, b->stream), R)) return LSMGPU_ERR_CUDA;
  }
  if (sync && !cuda_ok(cudaStreamSynchronize(b->stream), R)) return LSMGPU_ERR_CUDA;
  return LSMGPU_SUCCESS;
}

void* lsmgpu_batch_stream(lsmgpu_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"
