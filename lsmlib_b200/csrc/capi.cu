// capi.cu -- extern "C" entry points: the reference-compatible toolbox
// routines (Part 1 of include/lsmgpu/lsmgpu.h) and the basic extension API.
//
// Every routine follows the same shape: read the box pointers, validate them
// against the stencil the routine reads, map each array to a device pointer
// (in place or staged), launch the kernel on the calling thread's stream,
// and finish (copy back staged outputs, synchronise when required).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "capi_common.h"
#include "launch.h"
#include "stencil.cuh"

namespace lsmgpu {

// ---------------------------------------------------------------------------
// thread-local state
// ---------------------------------------------------------------------------
namespace {
thread_local int t_err = LSMGPU_SUCCESS;
thread_local std::string t_msg;
thread_local std::string t_msg_out;
thread_local cudaStream_t t_stream = nullptr;
int g_sync = 0;
int g_fp_mode = LSMGPU_FP_STRICT;
}  // namespace

void set_error(int code, const std::string& msg) {
  t_err = code;
  t_msg = msg;
  if (getenv("LSMGPU_VERBOSE")) fprintf(stderr, "lsmgpu: %s\n", msg.c_str());
}
void clear_error() {
  t_err = LSMGPU_SUCCESS;
  t_msg.clear();
}
bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(LSMGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}
cudaStream_t cur_stream() { return t_stream; }
bool sync_mode() { return g_sync != 0; }
int fp_mode() { return g_fp_mode; }

// ---------------------------------------------------------------------------
// boxes
// ---------------------------------------------------------------------------
Box box_from(const int* ilo, const int* ihi, const int* jlo, const int* jhi,
             const int* klo, const int* khi) {
  Box b;
  b.lo[0] = *ilo; b.lo[1] = *jlo; b.lo[2] = *klo;
  b.n[0] = *ihi - *ilo + 1; b.n[1] = *jhi - *jlo + 1; b.n[2] = *khi - *klo + 1;
  return b;
}
FillBox fill_from(const int* ilo, const int* ihi, const int* jlo,
                  const int* jhi, const int* klo, const int* khi) {
  FillBox f;
  f.lo[0] = *ilo; f.lo[1] = *jlo; f.lo[2] = *klo;
  f.hi[0] = *ihi; f.hi[1] = *jhi; f.hi[2] = *khi;
  return f;
}
static bool fb_empty(const FillBox& fb) {
  return fb.hi[0] < fb.lo[0] || fb.hi[1] < fb.lo[1] || fb.hi[2] < fb.lo[2];
}
bool box_valid(const Box& b, const char* what, const char* routine) {
  if (b.n[0] < 1 || b.n[1] < 1 || b.n[2] < 1) {
    set_error(LSMGPU_ERR_INVALID_BOX,
              std::string(routine) + ": empty ghost box for " + what);
    return false;
  }
  return true;
}
bool covers3(const Box& b, const FillBox& fb, const int w[3], const char* what,
             const char* routine) {
  for (int d = 0; d < 3; d++) {
    if ((long)fb.lo[d] - w[d] < (long)b.lo[d] ||
        (long)fb.hi[d] + w[d] > (long)b.hi(d)) {
      char buf[256];
      snprintf(buf, sizeof buf,
               "%s: ghost box of %s [%d,%d] along axis %d does not cover the "
               "fill box [%d,%d] widened by %d",
               routine, what, b.lo[d], b.hi(d), d, fb.lo[d], fb.hi[d], w[d]);
      set_error(LSMGPU_ERR_INVALID_BOX, buf);
      return false;
    }
  }
  return true;
}
bool covers(const Box& b, const FillBox& fb, int w, const char* what,
            const char* routine) {
  const int ww[3] = {w, w, w};
  return covers3(b, fb, ww, what, routine);
}

// ---------------------------------------------------------------------------
// scratch pool
// ---------------------------------------------------------------------------
namespace {
constexpr int kMaxDevices = 64;
// freed memory the pool keeps mapped between calls (the distance function
// of a 256^3 grid takes 1.4 GB of scratch)
constexpr unsigned long long kRetainBytes = 8ULL << 30;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};

cudaMemPool_t device_pool(int dev) {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    unsigned long long keep = kRetainBytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pool[dev] = pool;
  }
  return g_pool[dev];
}
}  // namespace

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool = dev >= 0 && dev < kMaxDevices ? device_pool(dev) : nullptr;
  // the device's default pool when no pool of our own can be made
  return pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaMallocAsync(p, bytes, st);
}

// ---------------------------------------------------------------------------
// staging
// ---------------------------------------------------------------------------
bool is_device_pointer(const void* p) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void* Staging::add(const void* p, const Box& b, int elem, Role role,
                   const char* what, const char* routine) {
  if (!p) {
    set_error(LSMGPU_ERR_NULL_POINTER,
              std::string(routine) + ": null pointer for " + what);
    return nullptr;
  }
  Item it{const_cast<void*>(p), nullptr, (size_t)b.count() * (size_t)elem,
          role, false};
  if (is_device_pointer(p)) {
    it.dev = it.host;
  } else {
    it.staged = true;
    staged_ = true;
    if (!cuda_ok(pool_alloc(&it.dev, it.bytes, st_), "cudaMallocFromPoolAsync")) {
      set_error(LSMGPU_ERR_ALLOC, std::string(routine) +
                                      ": cannot allocate staging buffer for " +
                                      what);
      return nullptr;
    }
    // outputs are copied in too (cells outside the fill box keep their
    // values), unless the routine writes every cell
    if (role != kOutFull &&
        !cuda_ok(cudaMemcpyAsync(it.dev, it.host, it.bytes,
                                 cudaMemcpyHostToDevice, st_),
                 "cudaMemcpyAsync(H2D)")) {
      cudaFreeAsync(it.dev, st_);
      return nullptr;
    }
  }
  items_.push_back(it);
  return it.dev;
}

bool Staging::finish(const char* routine) {
  done_ = true;
  bool ok = true;
  for (auto& it : items_) {
    if (it.staged && (it.role & kOut) && ok)
      ok = cuda_ok(cudaMemcpyAsync(it.host, it.dev, it.bytes,
                                   cudaMemcpyDeviceToHost, st_),
                   "cudaMemcpyAsync(D2H)");
  }
  for (auto& it : items_)
    if (it.staged) cudaFreeAsync(it.dev, st_);
  items_.clear();
  if (staged_ || sync_mode())
    ok = cuda_ok(cudaStreamSynchronize(st_), routine) && ok;
  return ok;
}

Staging::~Staging() {
  if (!done_)
    for (auto& it : items_)
      if (it.staged) cudaFreeAsync(it.dev, st_);
}

ReduceScratch::ReduceScratch(cudaStream_t st, int n) : st_(st), n_(n) {
  if (pool_alloc((void**)&p_, sizeof(double) * (size_t)(n + 1), st) != cudaSuccess) {
    cudaGetLastError();
    p_ = nullptr;
    set_error(LSMGPU_ERR_ALLOC, "cannot allocate reduction scratch");
  }
}
ReduceScratch::~ReduceScratch() {
  if (p_) cudaFreeAsync(p_, st_);
}

}  // namespace lsmgpu

using namespace lsmgpu;

// ---------------------------------------------------------------------------
// helpers for the entry points
// ---------------------------------------------------------------------------
#define BOX(p) box_from(ilo_##p, ihi_##p, jlo_##p, jhi_##p, klo_##p, khi_##p)
#define FB() fill_from(ilo_fb, ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb)
#define IB() fill_from(ilo_ib, ihi_ib, jlo_ib, jhi_ib, klo_ib, khi_ib)
#define NULLCHK(...)                                                       \
  do {                                                                     \
    const void* ps_[] = {__VA_ARGS__};                                     \
    for (const void* p_ : ps_)                                             \
      if (!p_) {                                                           \
        set_error(LSMGPU_ERR_NULL_POINTER,                                 \
                  std::string(R) + ": null argument pointer");             \
        return;                                                            \
      }                                                                    \
  } while (0)

static const int kReal = (int)sizeof(LSMLIB_REAL);

// Shared body of the plus/minus derivative routines.
static void hj_plus_minus(const char* R, int scheme, LSMLIB_REAL* const op[3],
                          const Box& gp, LSMLIB_REAL* const om[3],
                          const Box& gm, const LSMLIB_REAL* phi,
                          const Box& gphi, const FillBox& fb,
                          const LSMLIB_REAL* dx, const LSMLIB_REAL* dy,
                          const LSMLIB_REAL* dz) {
  clear_error();
  if (fb_empty(fb)) return;
  const int w = scheme_width(scheme);
  if (!box_valid(gp, "grad_phi_plus", R) || !box_valid(gm, "grad_phi_minus", R) ||
      !box_valid(gphi, "phi", R) || !covers(gp, fb, 0, "grad_phi_plus", R) ||
      !covers(gm, fb, 0, "grad_phi_minus", R) || !covers(gphi, fb, w, "phi", R))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  void *dp[3], *dm[3];
  const char* np[3] = {"phi_x_plus", "phi_y_plus", "phi_z_plus"};
  const char* nm[3] = {"phi_x_minus", "phi_y_minus", "phi_z_minus"};
  for (int d = 0; d < 3; d++) {
    if (!(dp[d] = s.add(op[d], gp, kReal, kOut, np[d], R))) return;
    if (!(dm[d] = s.add(om[d], gm, kReal, kOut, nm[d], R))) return;
  }
  const void* dphi = s.add(phi, gphi, kReal, kIn, "phi", R);
  if (!dphi) return;
  const double inv[3] = {1.0 / *dx, 1.0 / *dy, 1.0 / *dz};
  if (!cuda_ok(launch_hj_plus_minus(scheme, kReal, dp, gp, dm, gm, dphi, gphi,
                                    fb, inv, st),
               R))
    return;
  s.finish(R);
}

static void hj_upwind(const char* R, int scheme, LSMLIB_REAL* const o[3],
                      const Box& go, const LSMLIB_REAL* phi, const Box& gphi,
                      const LSMLIB_REAL* const v[3], const Box& gv,
                      const FillBox& fb, const LSMLIB_REAL* dx,
                      const LSMLIB_REAL* dy, const LSMLIB_REAL* dz) {
  clear_error();
  if (fb_empty(fb)) return;
  const int w = scheme_width(scheme);
  if (!box_valid(go, "grad_phi", R) || !box_valid(gphi, "phi", R) ||
      !box_valid(gv, "vel", R) || !covers(go, fb, 0, "grad_phi", R) ||
      !covers(gphi, fb, w, "phi", R) || !covers(gv, fb, 0, "vel", R))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  void* dout[3];
  const void* dv[3];
  const char* no[3] = {"phi_x", "phi_y", "phi_z"};
  const char* nv[3] = {"vel_x", "vel_y", "vel_z"};
  for (int d = 0; d < 3; d++) {
    if (!(dout[d] = s.add(o[d], go, kReal, kOut, no[d], R))) return;
    if (!(dv[d] = s.add(v[d], gv, kReal, kIn, nv[d], R))) return;
  }
  const void* dphi = s.add(phi, gphi, kReal, kIn, "phi", R);
  if (!dphi) return;
  const double inv[3] = {1.0 / *dx, 1.0 / *dy, 1.0 / *dz};
  if (!cuda_ok(launch_hj_upwind(scheme, kReal, dout, go, dphi, gphi, dv, gv, fb,
                                inv, st),
               R))
    return;
  s.finish(R);
}

// Arguments common to the plus/minus derivative prototypes.
#define PM_ARGS                                                             \
  LSMLIB_REAL *phi_x_plus, LSMLIB_REAL *phi_y_plus, LSMLIB_REAL *phi_z_plus, \
      LSMGPU_BOX6(gp), LSMLIB_REAL *phi_x_minus, LSMLIB_REAL *phi_y_minus,   \
      LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(gm), const LSMLIB_REAL *phi,     \
      LSMGPU_BOX6(phi)
#define PM_CALL(name, scheme)                                                \
  LSMLIB_REAL* const op_[3] = {phi_x_plus, phi_y_plus, phi_z_plus};          \
  LSMLIB_REAL* const om_[3] = {phi_x_minus, phi_y_minus, phi_z_minus};       \
  const char* R = name;                                                      \
  NULLCHK(ilo_gp, ihi_gp, jlo_gp, jhi_gp, klo_gp, khi_gp, ilo_gm, ihi_gm,    \
          jlo_gm, jhi_gm, klo_gm, khi_gm, ilo_phi, ihi_phi, jlo_phi,         \
          jhi_phi, klo_phi, khi_phi, ilo_fb, ihi_fb, jlo_fb, jhi_fb, klo_fb, \
          khi_fb, dx, dy, dz);                                               \
  hj_plus_minus(R, scheme, op_, BOX(gp), om_, BOX(gm), phi, BOX(phi), FB(),  \
                dx, dy, dz)
#define UP_ARGS                                                              \
  LSMLIB_REAL *phi_x, LSMLIB_REAL *phi_y, LSMLIB_REAL *phi_z, LSMGPU_BOX6(g), \
      const LSMLIB_REAL *phi, LSMGPU_BOX6(phi), const LSMLIB_REAL *vel_x,     \
      const LSMLIB_REAL *vel_y, const LSMLIB_REAL *vel_z, LSMGPU_BOX6(v)
#define UP_CALL(name, scheme)                                                \
  LSMLIB_REAL* const o_[3] = {phi_x, phi_y, phi_z};                          \
  const LSMLIB_REAL* const v_[3] = {vel_x, vel_y, vel_z};                    \
  const char* R = name;                                                      \
  NULLCHK(ilo_g, ihi_g, jlo_g, jhi_g, klo_g, khi_g, ilo_phi, ihi_phi,        \
          jlo_phi, jhi_phi, klo_phi, khi_phi, ilo_v, ihi_v, jlo_v, jhi_v,    \
          klo_v, khi_v, ilo_fb, ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb, dx,  \
          dy, dz);                                                           \
  hj_upwind(R, scheme, o_, BOX(g), phi, BOX(phi), v_, BOX(v), FB(), dx, dy, dz)

#define SCR(p) LSMLIB_REAL *p, LSMGPU_BOX6(p)
#define FB6 LSMGPU_BOX6(fb)
#define DXYZ const LSMLIB_REAL *dx, const LSMLIB_REAL *dy, const LSMLIB_REAL *dz

extern "C" {

void lsm3dhjeno1_(PM_ARGS, SCR(D1), FB6, DXYZ) { PM_CALL("LSM3D_HJ_ENO1", kENO1); }
void lsm3dhjeno2_(PM_ARGS, SCR(D1), SCR(D2), FB6, DXYZ) {
  PM_CALL("LSM3D_HJ_ENO2", kENO2);
}
void lsm3dhjeno3_(PM_ARGS, SCR(D1), SCR(D2), SCR(D3), FB6, DXYZ) {
  PM_CALL("LSM3D_HJ_ENO3", kENO3);
}
void lsm3dhjweno5_(PM_ARGS, SCR(D1), FB6, DXYZ) {
  PM_CALL("LSM3D_HJ_WENO5", kWENO5);
}
void lsm3dupwindhjeno1_(UP_ARGS, SCR(D1), FB6, DXYZ) {
  UP_CALL("LSM3D_UPWIND_HJ_ENO1", kENO1);
}
void lsm3dupwindhjeno2_(UP_ARGS, SCR(D1), SCR(D2), FB6, DXYZ) {
  UP_CALL("LSM3D_UPWIND_HJ_ENO2", kENO2);
}
void lsm3dupwindhjeno3_(UP_ARGS, SCR(D1), SCR(D2), SCR(D3), FB6, DXYZ) {
  UP_CALL("LSM3D_UPWIND_HJ_ENO3", kENO3);
}
void lsm3dupwindhjweno5_(UP_ARGS, SCR(D1), FB6, DXYZ) {
  UP_CALL("LSM3D_UPWIND_HJ_WENO5", kWENO5);
}

void lsm3dzerooutlevelseteqnrhs_(LSMLIB_REAL* lse_rhs, LSMGPU_BOX6(r)) {
  const char* R = "LSM3D_ZERO_OUT_LEVEL_SET_EQN_RHS";
  NULLCHK(ilo_r, ihi_r, jlo_r, jhi_r, klo_r, khi_r);
  clear_error();
  const Box gr = BOX(r);
  if (gr.n[0] < 1 || gr.n[1] < 1 || gr.n[2] < 1) return;  // nothing to zero
  cudaStream_t st = cur_stream();
  Staging s(st);
  void* d = s.add(lse_rhs, gr, kReal, kOut, "lse_rhs", R);
  if (!d) return;
  if (!cuda_ok(launch_fill(kReal, d, gr.count(), 0.0, st), R)) return;
  s.finish(R);
}

void lsm3daddadvectiontermtolserhs_(LSMLIB_REAL* lse_rhs, LSMGPU_BOX6(r),
                                    const LSMLIB_REAL* phi_x,
                                    const LSMLIB_REAL* phi_y,
                                    const LSMLIB_REAL* phi_z, LSMGPU_BOX6(g),
                                    const LSMLIB_REAL* vel_x,
                                    const LSMLIB_REAL* vel_y,
                                    const LSMLIB_REAL* vel_z, LSMGPU_BOX6(v),
                                    FB6) {
  const char* R = "LSM3D_ADD_ADVECTION_TERM_TO_LSE_RHS";
  NULLCHK(ilo_r, ihi_r, jlo_r, jhi_r, klo_r, khi_r, ilo_g, ihi_g, jlo_g, jhi_g,
          klo_g, khi_g, ilo_v, ihi_v, jlo_v, jhi_v, klo_v, khi_v, ilo_fb,
          ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb);
  clear_error();
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  const Box gr = BOX(r), gg = BOX(g), gv = BOX(v);
  if (!covers(gr, fb, 0, "lse_rhs", R) || !covers(gg, fb, 0, "grad_phi", R) ||
      !covers(gv, fb, 0, "vel", R))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  void* dr = s.add(lse_rhs, gr, kReal, kInOut, "lse_rhs", R);
  if (!dr) return;
  const void *dg[3], *dv[3];
  const LSMLIB_REAL* hg[3] = {phi_x, phi_y, phi_z};
  const LSMLIB_REAL* hv[3] = {vel_x, vel_y, vel_z};
  for (int d = 0; d < 3; d++) {
    if (!(dg[d] = s.add(hg[d], gg, kReal, kIn, "grad_phi", R))) return;
    if (!(dv[d] = s.add(hv[d], gv, kReal, kIn, "vel", R))) return;
  }
  if (!cuda_ok(launch_add_advection(kReal, dr, gr, dg, gg, dv, gv, fb, st), R))
    return;
  s.finish(R);
}

static void add_normal(const char* R, LSMLIB_REAL* lse_rhs, const Box& gr,
                       const LSMLIB_REAL* const hp[3], const Box& gp,
                       const LSMLIB_REAL* const hm[3], const Box& gm,
                       const LSMLIB_REAL* vel_n, const Box* gv, double vconst,
                       const FillBox& fb) {
  clear_error();
  if (fb_empty(fb)) return;
  if (!covers(gr, fb, 0, "lse_rhs", R) || !covers(gp, fb, 0, "grad_phi_plus", R) ||
      !covers(gm, fb, 0, "grad_phi_minus", R) ||
      (gv && !covers(*gv, fb, 0, "vel_n", R)))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  void* dr = s.add(lse_rhs, gr, kReal, kInOut, "lse_rhs", R);
  if (!dr) return;
  const void *dp[3], *dm[3];
  for (int d = 0; d < 3; d++) {
    if (!(dp[d] = s.add(hp[d], gp, kReal, kIn, "grad_phi_plus", R))) return;
    if (!(dm[d] = s.add(hm[d], gm, kReal, kIn, "grad_phi_minus", R))) return;
  }
  const void* dv = nullptr;
  if (gv && !(dv = s.add(vel_n, *gv, kReal, kIn, "vel_n", R))) return;
  if (!cuda_ok(launch_add_normal(kReal, dr, gr, dp, gp, dm, gm, dv,
                                 gv ? *gv : gr, vconst, fb, st),
               R))
    return;
  s.finish(R);
}

void lsm3daddnormalveltermtolserhs_(
    LSMLIB_REAL* lse_rhs, LSMGPU_BOX6(r), const LSMLIB_REAL* phi_x_plus,
    const LSMLIB_REAL* phi_y_plus, const LSMLIB_REAL* phi_z_plus,
    LSMGPU_BOX6(gp), const LSMLIB_REAL* phi_x_minus,
    const LSMLIB_REAL* phi_y_minus, const LSMLIB_REAL* phi_z_minus,
    LSMGPU_BOX6(gm), const LSMLIB_REAL* vel_n, LSMGPU_BOX6(v), FB6) {
  const char* R = "LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS";
  NULLCHK(ilo_r, ihi_r, jlo_r, jhi_r, klo_r, khi_r, ilo_gp, ihi_gp, jlo_gp,
          jhi_gp, klo_gp, khi_gp, ilo_gm, ihi_gm, jlo_gm, jhi_gm, klo_gm,
          khi_gm, ilo_v, ihi_v, jlo_v, jhi_v, klo_v, khi_v, ilo_fb, ihi_fb,
          jlo_fb, jhi_fb, klo_fb, khi_fb);
  const LSMLIB_REAL* hp[3] = {phi_x_plus, phi_y_plus, phi_z_plus};
  const LSMLIB_REAL* hm[3] = {phi_x_minus, phi_y_minus, phi_z_minus};
  const Box gv = BOX(v);
  add_normal(R, lse_rhs, BOX(r), hp, BOX(gp), hm, BOX(gm), vel_n, &gv, 0.0,
             FB());
}

void lsm3daddconstnormalveltermtolserhs_(
    LSMLIB_REAL* lse_rhs, LSMGPU_BOX6(r), const LSMLIB_REAL* phi_x_plus,
    const LSMLIB_REAL* phi_y_plus, const LSMLIB_REAL* phi_z_plus,
    LSMGPU_BOX6(gp), const LSMLIB_REAL* phi_x_minus,
    const LSMLIB_REAL* phi_y_minus, const LSMLIB_REAL* phi_z_minus,
    LSMGPU_BOX6(gm), const LSMLIB_REAL* vel_n, FB6) {
  const char* R = "LSM3D_ADD_CONST_NORMAL_VEL_TERM_TO_LSE_RHS";
  NULLCHK(ilo_r, ihi_r, jlo_r, jhi_r, klo_r, khi_r, ilo_gp, ihi_gp, jlo_gp,
          jhi_gp, klo_gp, khi_gp, ilo_gm, ihi_gm, jlo_gm, jhi_gm, klo_gm,
          khi_gm, vel_n, ilo_fb, ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb);
  clear_error();
  // lsm_level_set_evolution3d.f.in:297: nothing to add when |F| < zero_tol
  if (!(fabs(*vel_n) >= Consts<LSMLIB_REAL>::zero_tol)) return;
  const LSMLIB_REAL* hp[3] = {phi_x_plus, phi_y_plus, phi_z_plus};
  const LSMLIB_REAL* hm[3] = {phi_x_minus, phi_y_minus, phi_z_minus};
  add_normal(R, lse_rhs, BOX(r), hp, BOX(gp), hm, BOX(gm), nullptr, nullptr,
             *vel_n, FB());
}

void lsm3dcomputereinitializationeqnrhs_(
    LSMLIB_REAL* reinit_rhs, LSMGPU_BOX6(r), const LSMLIB_REAL* phi,
    LSMGPU_BOX6(phi), const LSMLIB_REAL* phi0, LSMGPU_BOX6(phi0),
    const LSMLIB_REAL* phi_x_plus, const LSMLIB_REAL* phi_y_plus,
    const LSMLIB_REAL* phi_z_plus, LSMGPU_BOX6(gp),
    const LSMLIB_REAL* phi_x_minus, const LSMLIB_REAL* phi_y_minus,
    const LSMLIB_REAL* phi_z_minus, LSMGPU_BOX6(gm), FB6, DXYZ,
    const int* use_phi0_for_sgn) {
  const char* R = "LSM3D_COMPUTE_REINITIALIZATION_EQN_RHS";
  NULLCHK(ilo_r, ihi_r, jlo_r, jhi_r, klo_r, khi_r, ilo_phi, ihi_phi, jlo_phi,
          jhi_phi, klo_phi, khi_phi, ilo_phi0, ihi_phi0, jlo_phi0, jhi_phi0,
          klo_phi0, khi_phi0, ilo_gp, ihi_gp, jlo_gp, jhi_gp, klo_gp, khi_gp,
          ilo_gm, ihi_gm, jlo_gm, jhi_gm, klo_gm, khi_gm, ilo_fb, ihi_fb,
          jlo_fb, jhi_fb, klo_fb, khi_fb, dx, dy, dz, use_phi0_for_sgn);
  clear_error();
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  const Box gr = BOX(r), gphi = BOX(phi), gphi0 = BOX(phi0), gp = BOX(gp),
            gm = BOX(gm);
  const int use0 = *use_phi0_for_sgn;
  if (!covers(gr, fb, 0, "reinit_rhs", R) || !covers(gphi, fb, 0, "phi", R) ||
      (use0 == 1 && !covers(gphi0, fb, 0, "phi0", R)) ||
      !covers(gp, fb, 0, "grad_phi_plus", R) ||
      !covers(gm, fb, 0, "grad_phi_minus", R))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  void* dr = s.add(reinit_rhs, gr, kReal, kOut, "reinit_rhs", R);
  if (!dr) return;
  const void* dphi = s.add(phi, gphi, kReal, kIn, "phi", R);
  if (!dphi) return;
  // phi0 is only read when use_phi0_for_sgn == 1 (the reference reads it
  // nowhere else), so a null phi0 is accepted otherwise
  const void* dphi0 = dphi;
  if (use0 == 1 && !(dphi0 = s.add(phi0, gphi0, kReal, kIn, "phi0", R))) return;
  const LSMLIB_REAL* hp[3] = {phi_x_plus, phi_y_plus, phi_z_plus};
  const LSMLIB_REAL* hm[3] = {phi_x_minus, phi_y_minus, phi_z_minus};
  const void *dp[3], *dm[3];
  for (int d = 0; d < 3; d++) {
    if (!(dp[d] = s.add(hp[d], gp, kReal, kIn, "grad_phi_plus", R))) return;
    if (!(dm[d] = s.add(hm[d], gm, kReal, kIn, "grad_phi_minus", R))) return;
  }
  // lsm_reinitialization3d.f.in:140-141
  LSMLIB_REAL dx_sq = *dx > *dy ? *dx : *dy;
  dx_sq = dx_sq > *dz ? dx_sq : *dz;
  dx_sq = dx_sq * dx_sq;
  if (!cuda_ok(launch_reinit_rhs(kReal, dr, gr, dphi, gphi, dphi0,
                                 use0 == 1 ? gphi0 : gphi, dp, gp, dm, gm, fb,
                                 dx_sq, use0, st),
               R))
    return;
  s.finish(R);
}

void lsm3dcomputefieldextensioneqnrhs_(
    LSMLIB_REAL* rhs, LSMGPU_BOX6(r), const LSMLIB_REAL* S, LSMGPU_BOX6(S),
    const LSMLIB_REAL* phi, LSMGPU_BOX6(phi), const LSMLIB_REAL* S_x_upwind,
    const LSMLIB_REAL* S_y_upwind, const LSMLIB_REAL* S_z_upwind,
    LSMGPU_BOX6(gs), const LSMLIB_REAL* signed_normal_x,
    const LSMLIB_REAL* signed_normal_y, const LSMLIB_REAL* signed_normal_z,
    LSMGPU_BOX6(gn), FB6, DXYZ) {
  const char* R = "LSM3D_COMPUTE_FIELD_EXTENSION_EQN_RHS";
  (void)S; (void)ilo_S; (void)ihi_S; (void)jlo_S; (void)jhi_S; (void)klo_S;
  (void)khi_S;
  NULLCHK(ilo_r, ihi_r, jlo_r, jhi_r, klo_r, khi_r, ilo_phi, ihi_phi, jlo_phi,
          jhi_phi, klo_phi, khi_phi, ilo_gs, ihi_gs, jlo_gs, jhi_gs, klo_gs,
          khi_gs, ilo_gn, ihi_gn, jlo_gn, jhi_gn, klo_gn, khi_gn, ilo_fb,
          ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb, dx, dy, dz);
  clear_error();
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  const Box gr = BOX(r), gphi = BOX(phi), ggs = BOX(gs), ggn = BOX(gn);
  if (!covers(gr, fb, 0, "rhs", R) || !covers(gphi, fb, 1, "phi", R) ||
      !covers(ggs, fb, 0, "grad_S_upwind", R) ||
      !covers(ggn, fb, 0, "signed_normal", R))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  void* dr = s.add(rhs, gr, kReal, kOut, "rhs", R);
  if (!dr) return;
  const void* dphi = s.add(phi, gphi, kReal, kIn, "phi", R);
  if (!dphi) return;
  const LSMLIB_REAL* hs[3] = {S_x_upwind, S_y_upwind, S_z_upwind};
  const LSMLIB_REAL* hn[3] = {signed_normal_x, signed_normal_y, signed_normal_z};
  const void *ds[3], *dn[3];
  for (int d = 0; d < 3; d++) {
    if (!(ds[d] = s.add(hs[d], ggs, kReal, kIn, "grad_S_upwind", R))) return;
    if (!(dn[d] = s.add(hn[d], ggn, kReal, kIn, "signed_normal", R))) return;
  }
  // lsm_field_extension3d.f:115
  LSMLIB_REAL m = *dx > *dy ? *dx : *dy;
  m = m > *dz ? m : *dz;
  const LSMLIB_REAL cutoff = 3.0 * m;
  if (!cuda_ok(launch_field_ext_rhs(kReal, dr, gr, dphi, gphi, ds, ggs, dn, ggn,
                                    fb, cutoff, st),
               R))
    return;
  s.finish(R);
}

void lsm3dcomputesignedunitnormal_(
    LSMLIB_REAL* normal_x, LSMLIB_REAL* normal_y, LSMLIB_REAL* normal_z,
    LSMGPU_BOX6(gn), const LSMLIB_REAL* phi_x, const LSMLIB_REAL* phi_y,
    const LSMLIB_REAL* phi_z, LSMGPU_BOX6(g), const LSMLIB_REAL* phi,
    LSMGPU_BOX6(phi), FB6, DXYZ) {
  const char* R = "LSM3D_COMPUTE_SIGNED_UNIT_NORMAL";
  NULLCHK(ilo_gn, ihi_gn, jlo_gn, jhi_gn, klo_gn, khi_gn, ilo_g, ihi_g, jlo_g,
          jhi_g, klo_g, khi_g, ilo_phi, ihi_phi, jlo_phi, jhi_phi, klo_phi,
          khi_phi, ilo_fb, ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb, dx, dy, dz);
  clear_error();
  const FillBox fb = FB();
  if (fb_empty(fb)) return;
  const Box ggn = BOX(gn), gg = BOX(g), gphi = BOX(phi);
  if (!covers(ggn, fb, 0, "normal", R) || !covers(gg, fb, 0, "grad_phi", R) ||
      !covers(gphi, fb, 0, "phi", R))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  LSMLIB_REAL* hn[3] = {normal_x, normal_y, normal_z};
  const LSMLIB_REAL* hg[3] = {phi_x, phi_y, phi_z};
  void* dn[3];
  const void* dg[3];
  for (int d = 0; d < 3; d++) {
    if (!(dn[d] = s.add(hn[d], ggn, kReal, kOut, "normal", R))) return;
    if (!(dg[d] = s.add(hg[d], gg, kReal, kIn, "grad_phi", R))) return;
  }
  const void* dphi = s.add(phi, gphi, kReal, kIn, "phi", R);
  if (!dphi) return;
  LSMLIB_REAL dx_sq = *dx > *dy ? *dx : *dy;
  dx_sq = dx_sq > *dz ? dx_sq : *dz;
  dx_sq = dx_sq * dx_sq;
  if (!cuda_ok(launch_signed_normal(kReal, dn, ggn, dg, gg, dphi, gphi, fb,
                                    dx_sq, st),
               R))
    return;
  s.finish(R);
}

// ---- TVD Runge-Kutta -------------------------------------------------------
static void rk_call(const char* R, int kind, LSMLIB_REAL* out, const Box& go,
                    const LSMLIB_REAL* us, const Box* gus,
                    const LSMLIB_REAL* uc, const Box& guc,
                    const LSMLIB_REAL* rhs, const Box& grhs, const FillBox& fb,
                    const LSMLIB_REAL* dt) {
  clear_error();
  if (fb_empty(fb)) return;
  if (!covers(go, fb, 0, "u_out", R) || !covers(guc, fb, 0, "u_cur", R) ||
      !covers(grhs, fb, 0, "rhs", R) || (gus && !covers(*gus, fb, 0, "u_stage", R)))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  void* dout = s.add(out, go, kReal, kOut, "u_out", R);
  if (!dout) return;
  const void* dus = nullptr;
  if (gus && !(dus = s.add(us, *gus, kReal, kIn, "u_stage", R))) return;
  const void* duc = s.add(uc, guc, kReal, kIn, "u_cur", R);
  if (!duc) return;
  const void* dr = s.add(rhs, grhs, kReal, kIn, "rhs", R);
  if (!dr) return;
  if (!cuda_ok(launch_rk(kReal, kind, dout, go, dus, gus ? *gus : guc, duc, guc,
                         dr, grhs, fb, *dt, nullptr, st),
               R))
    return;
  s.finish(R);
}

#define RK1_ARGS                                                         \
  LSMLIB_REAL *u_out, LSMGPU_BOX6(o), const LSMLIB_REAL *u_cur,          \
      LSMGPU_BOX6(c), const LSMLIB_REAL *rhs, LSMGPU_BOX6(r), FB6,       \
      const LSMLIB_REAL *dt
#define RK1_NULLCHK                                                          \
  NULLCHK(ilo_o, ihi_o, jlo_o, jhi_o, klo_o, khi_o, ilo_c, ihi_c, jlo_c,     \
          jhi_c, klo_c, khi_c, ilo_r, ihi_r, jlo_r, jhi_r, klo_r, khi_r,     \
          ilo_fb, ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb, dt)

void lsm3drk1step_(RK1_ARGS) {
  const char* R = "LSM3D_RK1_STEP";
  RK1_NULLCHK;
  rk_call(R, 1, u_out, BOX(o), nullptr, nullptr, u_cur, BOX(c), rhs, BOX(r),
          FB(), dt);
}
void lsm3dtvdrk2stage1_(RK1_ARGS) {
  const char* R = "LSM3D_TVD_RK2_STAGE1";
  RK1_NULLCHK;
  rk_call(R, 1, u_out, BOX(o), nullptr, nullptr, u_cur, BOX(c), rhs, BOX(r),
          FB(), dt);
}
void lsm3dtvdrk3stage1_(RK1_ARGS) {
  const char* R = "LSM3D_TVD_RK3_STAGE1";
  RK1_NULLCHK;
  rk_call(R, 1, u_out, BOX(o), nullptr, nullptr, u_cur, BOX(c), rhs, BOX(r),
          FB(), dt);
}

#define RK2_ARGS                                                         \
  LSMLIB_REAL *u_out, LSMGPU_BOX6(o), const LSMLIB_REAL *u_stage,        \
      LSMGPU_BOX6(s), const LSMLIB_REAL *u_cur, LSMGPU_BOX6(c),          \
      const LSMLIB_REAL *rhs, LSMGPU_BOX6(r), FB6, const LSMLIB_REAL *dt
#define RK2_CALL(name, kind)                                                 \
  const char* R = name;                                                      \
  NULLCHK(ilo_o, ihi_o, jlo_o, jhi_o, klo_o, khi_o, ilo_s, ihi_s, jlo_s,     \
          jhi_s, klo_s, khi_s, ilo_c, ihi_c, jlo_c, jhi_c, klo_c, khi_c,     \
          ilo_r, ihi_r, jlo_r, jhi_r, klo_r, khi_r, ilo_fb, ihi_fb, jlo_fb,  \
          jhi_fb, klo_fb, khi_fb, dt);                                       \
  const Box gs_ = BOX(s);                                                    \
  rk_call(R, kind, u_out, BOX(o), u_stage, &gs_, u_cur, BOX(c), rhs, BOX(r), \
          FB(), dt)

void lsm3dtvdrk2stage2_(RK2_ARGS) { RK2_CALL("LSM3D_TVD_RK2_STAGE2", 22); }
void lsm3dtvdrk3stage2_(RK2_ARGS) { RK2_CALL("LSM3D_TVD_RK3_STAGE2", 32); }
void lsm3dtvdrk3stage3_(RK2_ARGS) { RK2_CALL("LSM3D_TVD_RK3_STAGE3", 33); }

// ---- reductions --------------------------------------------------------------
// Result is written to a host or device scalar; a host scalar makes the call
// synchronous.
static void deliver(const char* R, LSMLIB_REAL* out, const double* dres,
                    cudaStream_t st, Staging& s) {
  if (is_device_pointer(out)) {
    if (!cuda_ok(cudaMemcpyAsync(out, dres, sizeof(double),
                                 cudaMemcpyDeviceToDevice, st),
                 R))
      return;
    s.finish(R);
  } else {
    double v = 0.0;
    if (!cuda_ok(cudaMemcpyAsync(&v, dres, sizeof(double),
                                 cudaMemcpyDeviceToHost, st),
                 R))
      return;
    if (!s.finish(R)) return;
    if (!cuda_ok(cudaStreamSynchronize(st), R)) return;
    *out = v;
  }
}

void lsm3dmaxnormdiff_(LSMLIB_REAL* max_norm_diff, const LSMLIB_REAL* field1,
                       LSMGPU_BOX6(f1), const LSMLIB_REAL* field2,
                       LSMGPU_BOX6(f2), LSMGPU_BOX6(ib)) {
  const char* R = "LSM3D_MAX_NORM_DIFF";
  NULLCHK(max_norm_diff, ilo_f1, ihi_f1, jlo_f1, jhi_f1, klo_f1, khi_f1,
          ilo_f2, ihi_f2, jlo_f2, jhi_f2, klo_f2, khi_f2, ilo_ib, ihi_ib,
          jlo_ib, jhi_ib, klo_ib, khi_ib);
  clear_error();
  const FillBox ib = IB();
  const Box g1 = BOX(f1), g2 = BOX(f2);
  // the reference reads the first cell of the include box unconditionally
  // (lsm_utilities3d.f.in:57), so an empty include box is rejected
  if (fb_empty(ib)) {
    set_error(LSMGPU_ERR_INVALID_BOX, std::string(R) + ": empty include box");
    return;
  }
  if (!covers(g1, ib, 0, "field1", R) || !covers(g2, ib, 0, "field2", R)) return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  const void* d1 = s.add(field1, g1, kReal, kIn, "field1", R);
  if (!d1) return;
  const void* d2 = s.add(field2, g2, kReal, kIn, "field2", R);
  if (!d2) return;
  ReduceScratch scr(st, reduce_partials_needed(ib));
  if (!scr.ok()) return;
  if (!cuda_ok(launch_max_norm_diff(kReal, d1, g1, d2, g2, ib, scr.partials(),
                                    scr.result(), st),
               R))
    return;
  deliver(R, max_norm_diff, scr.result(), st, s);
}

void lsm3dcomputestableadvectiondt_(LSMLIB_REAL* dt, const LSMLIB_REAL* vel_x,
                                    const LSMLIB_REAL* vel_y,
                                    const LSMLIB_REAL* vel_z, LSMGPU_BOX6(v),
                                    LSMGPU_BOX6(ib), DXYZ,
                                    const LSMLIB_REAL* cfl_number) {
  const char* R = "LSM3D_COMPUTE_STABLE_ADVECTION_DT";
  NULLCHK(dt, ilo_v, ihi_v, jlo_v, jhi_v, klo_v, khi_v, ilo_ib, ihi_ib, jlo_ib,
          jhi_ib, klo_ib, khi_ib, dx, dy, dz, cfl_number);
  clear_error();
  const FillBox ib = IB();
  const Box gv = BOX(v);
  if (!fb_empty(ib) && !covers(gv, ib, 0, "vel", R)) return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  const LSMLIB_REAL* hv[3] = {vel_x, vel_y, vel_z};
  const void* dv[3];
  for (int d = 0; d < 3; d++)
    if (!(dv[d] = s.add(hv[d], gv, kReal, kIn, "vel", R))) return;
  FillBox ibr = ib;
  if (fb_empty(ib)) ibr.hi[0] = ibr.lo[0] - 1;  // zero cells: max stays -1
  ReduceScratch scr(st, reduce_partials_needed(ibr));
  if (!scr.ok()) return;
  const double inv[3] = {1.0 / *dx, 1.0 / *dy, 1.0 / *dz};
  if (!cuda_ok(launch_stable_advection_dt(kReal, dv, gv, ibr, inv, *cfl_number,
                                          scr.partials(), scr.result(), st),
               R))
    return;
  deliver(R, dt, scr.result(), st, s);
}

static void normal_dt(const char* R, LSMLIB_REAL* dt, const LSMLIB_REAL* vel_n,
                      const Box* gv, double vconst,
                      const LSMLIB_REAL* const hp[3], const Box& gp,
                      const LSMLIB_REAL* const hm[3], const Box& gm,
                      const FillBox& ib, const LSMLIB_REAL* dx,
                      const LSMLIB_REAL* dy, const LSMLIB_REAL* dz,
                      const LSMLIB_REAL* cfl) {
  clear_error();
  const bool empty = fb_empty(ib);
  if (!empty && (!covers(gp, ib, 0, "grad_phi_plus", R) ||
                 !covers(gm, ib, 0, "grad_phi_minus", R) ||
                 (gv && !covers(*gv, ib, 0, "vel_n", R))))
    return;
  cudaStream_t st = cur_stream();
  Staging s(st);
  const void *dp[3], *dm[3];
  for (int d = 0; d < 3; d++) {
    if (!(dp[d] = s.add(hp[d], gp, kReal, kIn, "grad_phi_plus", R))) return;
    if (!(dm[d] = s.add(hm[d], gm, kReal, kIn, "grad_phi_minus", R))) return;
  }
  const void* dv = nullptr;
  if (gv && !(dv = s.add(vel_n, *gv, kReal, kIn, "vel_n", R))) return;
  FillBox ibr = ib;
  if (empty) ibr.hi[0] = ibr.lo[0] - 1;
  ReduceScratch scr(st, reduce_partials_needed(ibr));
  if (!scr.ok()) return;
  // lsm_utilities3d.f.in:384-385
  LSMLIB_REAL m = *dx > *dy ? *dx : *dy;
  m = m > *dz ? m : *dz;
  const double inv[3] = {1.0 / *dx, 1.0 / *dy, 1.0 / *dz};
  if (!cuda_ok(launch_stable_normal_dt(kReal, dv, gv ? *gv : gp, vconst, dp, gp,
                                       dm, gm, ibr, inv, m * m, *cfl,
                                       scr.partials(), scr.result(), st),
               R))
    return;
  deliver(R, dt, scr.result(), st, s);
}

void lsm3dcomputestablenormalveldt_(
    LSMLIB_REAL* dt, const LSMLIB_REAL* vel_n, LSMGPU_BOX6(v),
    const LSMLIB_REAL* phi_x_plus, const LSMLIB_REAL* phi_y_plus,
    const LSMLIB_REAL* phi_z_plus, LSMGPU_BOX6(gp),
    const LSMLIB_REAL* phi_x_minus, const LSMLIB_REAL* phi_y_minus,
    const LSMLIB_REAL* phi_z_minus, LSMGPU_BOX6(gm), LSMGPU_BOX6(ib), DXYZ,
    const LSMLIB_REAL* cfl_number) {
  const char* R = "LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT";
  NULLCHK(dt, ilo_v, ihi_v, jlo_v, jhi_v, klo_v, khi_v, ilo_gp, ihi_gp, jlo_gp,
          jhi_gp, klo_gp, khi_gp, ilo_gm, ihi_gm, jlo_gm, jhi_gm, klo_gm,
          khi_gm, ilo_ib, ihi_ib, jlo_ib, jhi_ib, klo_ib, khi_ib, dx, dy, dz,
          cfl_number);
  const LSMLIB_REAL* hp[3] = {phi_x_plus, phi_y_plus, phi_z_plus};
  const LSMLIB_REAL* hm[3] = {phi_x_minus, phi_y_minus, phi_z_minus};
  const Box gv = BOX(v);
  normal_dt(R, dt, vel_n, &gv, 0.0, hp, BOX(gp), hm, BOX(gm), IB(), dx, dy, dz,
            cfl_number);
}

void lsm3dcomputestableconstnormalveldt_(
    LSMLIB_REAL* dt, const LSMLIB_REAL* vel_n, const LSMLIB_REAL* phi_x_plus,
    const LSMLIB_REAL* phi_y_plus, const LSMLIB_REAL* phi_z_plus,
    LSMGPU_BOX6(gp), const LSMLIB_REAL* phi_x_minus,
    const LSMLIB_REAL* phi_y_minus, const LSMLIB_REAL* phi_z_minus,
    LSMGPU_BOX6(gm), LSMGPU_BOX6(ib), DXYZ, const LSMLIB_REAL* cfl_number) {
  const char* R = "LSM3D_COMPUTE_STABLE_CONST_NORMAL_VEL_DT";
  NULLCHK(dt, vel_n, ilo_gp, ihi_gp, jlo_gp, jhi_gp, klo_gp, khi_gp, ilo_gm,
          ihi_gm, jlo_gm, jhi_gm, klo_gm, khi_gm, ilo_ib, ihi_ib, jlo_ib,
          jhi_ib, klo_ib, khi_ib, dx, dy, dz, cfl_number);
  const LSMLIB_REAL* hp[3] = {phi_x_plus, phi_y_plus, phi_z_plus};
  const LSMLIB_REAL* hm[3] = {phi_x_minus, phi_y_minus, phi_z_minus};
  normal_dt(R, dt, nullptr, nullptr, *vel_n, hp, BOX(gp), hm, BOX(gm), IB(), dx,
            dy, dz, cfl_number);
}

// ---- boundary conditions -------------------------------------------------------
static void bc_call(const char* R, int copy, LSMLIB_REAL* phi, const Box& gb,
                    const FillBox& fb, const int* face) {
  clear_error();
  const int f = *face;
  // the reference ignores indices outside 0..5 (no branch taken)
  if (f < 0 || f > 5) return;
  const int d = f / 2;
  if (!box_valid(gb, "phi", R) || !covers(gb, fb, 0, "phi", R)) return;
  // linear extrapolation reads two fill-box layers next to the face
  if (fb.hi[d] - fb.lo[d] + 1 < (copy ? 1 : 2)) {
    set_error(LSMGPU_ERR_INVALID_BOX,
              std::string(R) + ": fill box too thin along the face normal");
    return;
  }
  cudaStream_t st = cur_stream();
  Staging s(st);
  void* dphi = s.add(phi, gb, kReal, kInOut, "phi", R);
  if (!dphi) return;
  if (!cuda_ok(launch_bc(kReal, copy, dphi, gb, fb, f, st), R)) return;
  s.finish(R);
}

#define BC_ARGS \
  LSMLIB_REAL *phi, LSMGPU_BOX6(gb), FB6, const int *bdry_location_idx
#define BC_CALL(name, copy)                                                  \
  const char* R = name;                                                      \
  NULLCHK(phi, ilo_gb, ihi_gb, jlo_gb, jhi_gb, klo_gb, khi_gb, ilo_fb,       \
          ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb, bdry_location_idx);        \
  bc_call(R, copy, phi, BOX(gb), FB(), bdry_location_idx)

void lsm3dlinearextrapolation_(BC_ARGS) { BC_CALL("LSM3D_LINEAR_EXTRAPOLATION", 0); }
void lsm3dcopyextrapolation_(BC_ARGS) { BC_CALL("LSM3D_COPY_EXTRAPOLATION", 1); }
void lsm3dhomogeneousneumanneno1_(BC_ARGS) {
  BC_CALL("LSM3D_HOMOGENEOUS_NEUMANN_ENO1", 1);
}
void lsm3dhomogeneousneumanneno2_(BC_ARGS) {
  BC_CALL("LSM3D_HOMOGENEOUS_NEUMANN_ENO2", 1);
}
void lsm3dhomogeneousneumanneno3_(BC_ARGS) {
  BC_CALL("LSM3D_HOMOGENEOUS_NEUMANN_ENO3", 1);
}
void lsm3dhomogeneousneumannweno5_(BC_ARGS) {
  BC_CALL("LSM3D_HOMOGENEOUS_NEUMANN_WENO5", 1);
}

// ---------------------------------------------------------------------------
// Part 2: basic extension API
// ---------------------------------------------------------------------------
int lsmgpu_get_last_error(void) {
  int e = t_err;
  clear_error();
  return e;
}
int lsmgpu_peek_last_error(void) { return t_err; }
const char* lsmgpu_get_last_error_string(void) {
  t_msg_out = t_msg;
  return t_msg_out.c_str();
}
int lsmgpu_set_device(int device) {
  return cuda_ok(cudaSetDevice(device), "cudaSetDevice") ? LSMGPU_SUCCESS
                                                         : LSMGPU_ERR_CUDA;
}
int lsmgpu_set_stream(void* s) {
  t_stream = (cudaStream_t)s;
  return LSMGPU_SUCCESS;
}
void* lsmgpu_get_stream(void) { return (void*)t_stream; }
int lsmgpu_set_sync(int on) {
  g_sync = on ? 1 : 0;
  return LSMGPU_SUCCESS;
}
int lsmgpu_set_fp_mode(int mode) {
  if (mode != LSMGPU_FP_STRICT && mode != LSMGPU_FP_FAST) {
    set_error(LSMGPU_ERR_INVALID_VALUE, "lsmgpu_set_fp_mode: unknown mode");
    return LSMGPU_ERR_INVALID_VALUE;
  }
  g_fp_mode = mode;
  return LSMGPU_SUCCESS;
}
int lsmgpu_get_fp_mode(void) { return g_fp_mode; }
int lsmgpu_stream_synchronize(void) {
  return cuda_ok(cudaStreamSynchronize(t_stream), "cudaStreamSynchronize")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}
unsigned long long lsmgpu_kernel_launch_count(void) { return launch_counter(); }

void* lsmgpu_malloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error(LSMGPU_ERR_ALLOC, "lsmgpu_malloc: cudaMalloc failed");
    return nullptr;
  }
  return p;
}
int lsmgpu_free(void* p) {
  return cuda_ok(cudaFree(p), "cudaFree") ? LSMGPU_SUCCESS : LSMGPU_ERR_CUDA;
}
int lsmgpu_release_scratch(void) {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  bool ok = cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  for (int d = 0; d < kMaxDevices; d++)
    if (g_pool[d]) ok = cuda_ok(cudaMemPoolTrimTo(g_pool[d], 0), "cudaMemPoolTrimTo") && ok;
  return ok ? LSMGPU_SUCCESS : LSMGPU_ERR_CUDA;
}
void* lsmgpu_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error(LSMGPU_ERR_ALLOC, "lsmgpu_host_alloc: cudaMallocHost failed");
    return nullptr;
  }
  return p;
}
int lsmgpu_host_free(void* p) {
  return cuda_ok(cudaFreeHost(p), "cudaFreeHost") ? LSMGPU_SUCCESS
                                                  : LSMGPU_ERR_CUDA;
}
static int copy(void* d, const void* s, size_t n, cudaMemcpyKind k) {
  return cuda_ok(cudaMemcpyAsync(d, s, n, k, t_stream), "cudaMemcpyAsync") &&
                 cuda_ok(cudaStreamSynchronize(t_stream), "cudaStreamSynchronize")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}
int lsmgpu_memcpy_htod(void* d, const void* s, size_t n) {
  return copy(d, s, n, cudaMemcpyHostToDevice);
}
int lsmgpu_memcpy_dtoh(void* d, const void* s, size_t n) {
  return copy(d, s, n, cudaMemcpyDeviceToHost);
}
int lsmgpu_memcpy_dtod(void* d, const void* s, size_t n) {
  return copy(d, s, n, cudaMemcpyDeviceToDevice);
}
void* lsmgpu_event_create(void) {
  cudaEvent_t e = nullptr;
  if (!cuda_ok(cudaEventCreate(&e), "cudaEventCreate")) return nullptr;
  return (void*)e;
}
int lsmgpu_event_record(void* ev) {
  return cuda_ok(cudaEventRecord((cudaEvent_t)ev, t_stream), "cudaEventRecord")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}
int lsmgpu_event_elapsed_ms(void* a, void* b, float* ms) {
  if (!cuda_ok(cudaEventSynchronize((cudaEvent_t)b), "cudaEventSynchronize"))
    return LSMGPU_ERR_CUDA;
  return cuda_ok(cudaEventElapsedTime(ms, (cudaEvent_t)a, (cudaEvent_t)b),
                 "cudaEventElapsedTime")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}
int lsmgpu_event_destroy(void* ev) {
  return cuda_ok(cudaEventDestroy((cudaEvent_t)ev), "cudaEventDestroy")
             ? LSMGPU_SUCCESS
             : LSMGPU_ERR_CUDA;
}

}  // extern "C"
