// Shared host/device helpers for libnectb: error reporting and small utilities.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <type_traits>
#include <cuda_runtime.h>

#include "../../include/nectb.h"

namespace nectb {

// Records a message for nectb_last_error() and returns code.
int set_error(int code, const char* fmt, ...);
void clear_error();

inline int cuda_status(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return set_error(NECTB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return NECTB_OK;
}

// Checks the launch that was just enqueued (configuration errors only; the
// call never synchronises).
inline int launch_status(const char* what) { return cuda_status(cudaGetLastError(), what); }

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// The model shapes the fused kernels are instantiated for: 16 levels of F = 2
// or 4 features over D = 3 or 4 inputs, H = 2 or 3 hidden layers of 64.
// Calls fn(integral_constant D, F, H) for a supported shape and returns its
// result, else kUnsupportedShape.
constexpr int kUnsupportedShape = -1000;
template <typename Fn>
inline int dispatch_shape(int D, int F, int H, Fn&& fn) {
  using std::integral_constant;
#define NECTB_SHAPE(d, f, h) \
  if (D == d && F == f && H == h) return fn(integral_constant<int, d>{}, integral_constant<int, f>{}, integral_constant<int, h>{});
  NECTB_SHAPE(3, 2, 2) NECTB_SHAPE(3, 2, 3) NECTB_SHAPE(3, 4, 2) NECTB_SHAPE(3, 4, 3)
  NECTB_SHAPE(4, 2, 2) NECTB_SHAPE(4, 2, 3) NECTB_SHAPE(4, 4, 2) NECTB_SHAPE(4, 4, 3)
#undef NECTB_SHAPE
  return kUnsupportedShape;
}

// The current launch shapes and scheduling (nectb_set_tuning), copied under a lock.
NectbTuning current_tuning();

// Sets a kernel's dynamic shared memory and its L1/shared split.  An SM keeps
// one split while any block is resident, so a kernel that shares SMs with
// other launches (a capped background grid, serving queries) asks for a split
// with room for three ~51 KB blocks (164 of 228 KB, 92 KB left as L1):
// otherwise the split sized for it alone leaves no room for another kernel's
// blocks until the SM drains.  Kernels that own the GPU keep the driver's
// default split.
constexpr int kSharedCarveoutPercent = 72;
template <typename K>
inline void set_smem(K k, size_t bytes, bool shares_sms) {
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                       shares_sms ? kSharedCarveoutPercent : (int)cudaSharedmemCarveoutDefault);
}

// Records CUDA events around a kernel launch while profiling is enabled
// (nectb_profile_enable); slots are listed in include/nectb.h.
enum {
  kProfRayPrep = 0,
  kProfForward = 1,
  kProfBackward = 2,
  kProfAdam = 3,
  kProfSample = 4,
  kProfModel = 5,
  kProfScatter = 6,
  kProfOrder = 7,
  kProfSlice = 8
};
class ProfScope {
 public:
  ProfScope(int slot, cudaStream_t s);
  ~ProfScope();
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

 private:
  int slot_;
  cudaStream_t s_;
  void* a_;
};

}  // namespace nectb

#define NECTB_REQUIRE(cond, ...)                                        \
  do {                                                                  \
    if (!(cond)) return ::nectb::set_error(NECTB_ERR_INVALID, __VA_ARGS__); \
  } while (0)
