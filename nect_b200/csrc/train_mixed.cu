// Mixed-precision fused training step (fp16 tables, bf16 tcgen05 MLP).
#include "train_common.cuh"

namespace nectb {

int train_mixed(const NectbGeometry&, const GridDev&, const NectbMLP&, const void*, const float*, int,
                const TrainArgs&, Workspace, float*, float*, float*, float*, cudaStream_t) {
  return set_error(NECTB_ERR_INVALID, "mixed-precision path not built yet");
}

}  // namespace nectb
