// nectb_train_step_static: the fused training step with its scratch memory in
// a fixed device array owned by the library, for callers that cannot allocate
// device memory themselves.
//
// Who needs it: a host that reaches this library only through its C ABI and
// has no CUDA allocator of its own (a foreign-language runtime binding the
// .so), or a serving/training loop that must not call cudaMalloc at all
// (cudaMalloc synchronises the device and can fail under memory pressure in
// the middle of a run).  Such a caller passes only its inputs and outputs.
//
// The scratch is one file-scope __device__ array of kStaticScratchBytes
// (20 MiB + 4 KiB); every GPU that loads the library reserves it until the
// process exits.  Every call (with its device current) looks up the array's
// device address with cudaGetSymbolAddress; the first call on a device loads
// the module there, so make it before any stream capture.  All calls share the one array and it
// keeps the last call's contents: nectb_train_step clears what has to start
// at zero (scheduling cursors, error word, pixel slots) and overwrites the
// per-ray records, so results never depend on a previous call, but calls
// whose work overlaps on the GPU (different streams, or threads without
// ordering) race on the array and must be serialised by the caller.
#include "common.cuh"
#include "train_common.cuh"

extern "C" size_t nectb_train_workspace_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                              const NectbMLP* mlp, int32_t num_rays);

namespace nectb {
int validate_geometry(const NectbGeometry* g);
int train_step_loads_only(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                          const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                          float* grid_grad, float* mlp_grad, float* y_pred, float* loss, void* workspace,
                          size_t workspace_size, void* stream);
namespace {

constexpr size_t kStaticScratchBytes = (size_t(20) << 20) + 4096;
static __device__ __align__(256) unsigned char g_train_scratch[kStaticScratchBytes];

// Device address of g_train_scratch on the current device (the host-side
// symbol itself is not a device address).  Looked up on every call: the
// lookup allocates nothing, and a module reloaded after a context reset gets
// its new address.  It loads the module on the call's first use of the
// device, so that first call must come before any stream capture.
int scratch_address(void** out) {
  void* p = nullptr;
  if (int rc = cuda_status(cudaGetSymbolAddress(&p, g_train_scratch), "cudaGetSymbolAddress(g_train_scratch)"))
    return rc;
  *out = p;
  return NECTB_OK;
}

}  // namespace
}  // namespace nectb

extern "C" size_t nectb_train_static_scratch_bytes(void) { return nectb::kStaticScratchBytes; }

extern "C" int nectb_train_step_static(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                                       const void* grid_params, const float* mlp_params,
                                       const NectbTrainBatch* batch, float* grid_grad, float* mlp_grad,
                                       float* y_pred, float* loss, void* stream) {
  using namespace nectb;
  clear_error();
  NECTB_REQUIRE(geometry && grid && mlp && batch, "null description");
  if (int rc = validate_geometry(geometry)) return rc;
  const size_t need = nectb_train_workspace_bytes(geometry, grid, mlp, batch->num_rays);
  if (need > kStaticScratchBytes)
    return set_error(NECTB_ERR_TOO_LARGE,
                     "batch needs %zu bytes of scratch; the static scratch holds %zu (at most 262,144 rays on a "
                     "1024x1024 detector); use nectb_train_step with a caller workspace",
                     need, kStaticScratchBytes);
  void* scratch = nullptr;
  if (int rc = scratch_address(&scratch)) return rc;
  // the step of nectb_train_step on the static scratch, with plain loads (no
  // texture object: nothing is created on the caller's behalf)
  return train_step_loads_only(geometry, grid, mlp, grid_params, mlp_params, batch, grid_grad, mlp_grad, y_pred,
                               loss, scratch, kStaticScratchBytes, stream);
}

extern "C" const unsigned int* nectb_train_error_word(const NectbGeometry* geometry, int32_t num_rays,
                                                      const void* workspace) {
  using namespace nectb;
  clear_error();
  if (!geometry || num_rays <= 0) {
    set_error(NECTB_ERR_INVALID, "nectb_train_error_word: null geometry or num_rays <= 0");
    return nullptr;
  }
  if (validate_geometry(geometry) != NECTB_OK) return nullptr;
  void* ws = const_cast<void*>(workspace);
  if (!ws) {
    // the static scratch: only batches that nectb_train_step_static accepts have a word there
    if (nectb_train_workspace_bytes(geometry, nullptr, nullptr, num_rays) > kStaticScratchBytes) {
      set_error(NECTB_ERR_TOO_LARGE, "nectb_train_error_word: %d rays do not fit the static scratch", num_rays);
      return nullptr;
    }
    if (scratch_address(&ws) != NECTB_OK) return nullptr;
  }
  const int P = geometry->nDetector[0] * geometry->nDetector[1];
  return carve_workspace(ws, num_rays, P).counters + 2;
}
