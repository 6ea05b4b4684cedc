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

// Most warpgroups of the mixed forward on one SM (one block; 64 TMEM columns
// and at most 85 registers per thread each): NectbTuning::forward_blocks_per_sm
// and the re-projection's warpgroups_per_sm range over 1..kFwdMaxWarpgroups.
#ifndef NECTB_FWD_BLOCKS_PER_SM
#define NECTB_FWD_BLOCKS_PER_SM 6
#endif
constexpr int kFwdMaxWarpgroups = NECTB_FWD_BLOCKS_PER_SM;

// The model shapes the fused kernels are instantiated for, as (inputs D,
// features per level F, levels L, hidden layers H of width 64): 16 levels of
// 2 or 4 features over 3 or 4 inputs with 2 or 3 hidden layers (the
// benchmark workloads and their neighbours), and the reference's default
// static model, 19 levels of 4 features with 6 hidden layers
// (nect/cfg/static/hash_grid.yaml:1-13).  Calls fn(integral_constant D, F, L,
// H) for a supported shape and returns its result, else kUnsupportedShape.
constexpr int kUnsupportedShape = -1000;
template <typename Fn>
inline int dispatch_shape(int D, int F, int L, int H, Fn&& fn) {
  using std::integral_constant;
#define NECTB_SHAPE(d, f, l, h)                                                                                 \
  if (D == d && F == f && L == l && H == h)                                                                   \
    return fn(integral_constant<int, d>{}, integral_constant<int, f>{}, integral_constant<int, l>{},          \
              integral_constant<int, h>{});
  NECTB_SHAPE(3, 2, 16, 2) NECTB_SHAPE(3, 2, 16, 3) NECTB_SHAPE(3, 4, 16, 2) NECTB_SHAPE(3, 4, 16, 3)
  NECTB_SHAPE(4, 2, 16, 2) NECTB_SHAPE(4, 2, 16, 3) NECTB_SHAPE(4, 4, 16, 2) NECTB_SHAPE(4, 4, 16, 3)
  NECTB_SHAPE(3, 4, 19, 6)
#undef NECTB_SHAPE
  return kUnsupportedShape;
}

// Input row of the MLP for L levels of F features: IN values, padded with
// zeros to INP (a multiple of the MMA's K step of 16), held in KT tiles of 64
// columns (NCH 16-byte chunks of 8 bf16).
template <int L, int F>
struct InShape {
  static constexpr int IN = L * F;
  static constexpr int INP = (IN + 15) / 16 * 16;
  static constexpr int KT = (INP + 63) / 64;
  static constexpr int NCH = INP / 8;
  static_assert(KT <= 2, "at most 128 MLP inputs");
};

inline int input_padded(int n_input) { return (n_input + 15) / 16 * 16; }

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
