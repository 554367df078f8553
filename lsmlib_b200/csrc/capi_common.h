// capi_common.h -- host-side plumbing shared by the C ABI entry points:
// thread-local error state, the calling thread's stream, box validation and
// staging of host-resident arrays.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "../../include/lsmgpu/lsmgpu.h"

namespace lsmgpu {

// ---- error state (thread-local, like errno) -------------------------------
void set_error(int code, const std::string& msg);
void clear_error();
bool cuda_ok(cudaError_t e, const char* what);

// ---- per-thread configuration ---------------------------------------------
cudaStream_t cur_stream();
bool sync_mode();
int fp_mode();

// ---- boxes -----------------------------------------------------------------
Box box_from(const int* ilo, const int* ihi, const int* jlo, const int* jhi,
             const int* klo, const int* khi);
FillBox fill_from(const int* ilo, const int* ihi, const int* jlo,
                  const int* jhi, const int* klo, const int* khi);
bool box_valid(const Box& b, const char* what, const char* routine);
// fill box grown by ``w`` cells in every direction lies inside ``b``
bool covers(const Box& b, const FillBox& fb, int w, const char* what,
            const char* routine);
// fill box grown by w[d] cells along axis d lies inside ``b``
bool covers3(const Box& b, const FillBox& fb, const int w[3], const char* what,
             const char* routine);

// ---- device scratch -----------------------------------------------------------
// Stream-ordered allocation from the library's own memory pool on the
// current device.  Freed blocks stay mapped in the pool (up to a bound) for
// the next call, so a call that is repeated does not map its scratch again;
// lsmgpu_release_scratch() returns them to the driver.
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st);

// ---- staging ----------------------------------------------------------------
// kOutFull: an output the routine writes completely (no copy in)
enum Role { kIn = 1, kOut = 2, kInOut = 3, kOutFull = 6 };

bool is_device_pointer(const void* p);

// Collects the arrays of one call.  Device (or managed) pointers are used in
// place; host pointers are copied into stream-ordered device buffers before
// the kernels run and copied back (outputs) by finish().  A staged call is
// always synchronous; an in-place call is asynchronous unless sync mode is on.
class Staging {
 public:
  explicit Staging(cudaStream_t st) : st_(st) {}
  ~Staging();
  // returns the device pointer to use, or nullptr after recording an error
  void* add(const void* p, const Box& b, int elem, Role role, const char* what,
            const char* routine);
  bool any_staged() const { return staged_; }
  // copy staged outputs back, release buffers, synchronise if needed
  bool finish(const char* routine);

 private:
  struct Item {
    void* host;
    void* dev;
    size_t bytes;
    Role role;
    bool staged;
  };
  cudaStream_t st_;
  std::vector<Item> items_;
  bool staged_ = false;
  bool done_ = false;
};

// Device scratch for reductions: ``n`` doubles of partial maxima plus one
// result slot.  Stream-ordered allocation; freed by the destructor.
class ReduceScratch {
 public:
  ReduceScratch(cudaStream_t st, int n);
  ~ReduceScratch();
  double* partials() const { return p_; }
  double* result() const { return p_ ? p_ + n_ : nullptr; }
  bool ok() const { return p_ != nullptr; }

 private:
  cudaStream_t st_;
  int n_;
  double* p_ = nullptr;
};

}  // namespace lsmgpu
