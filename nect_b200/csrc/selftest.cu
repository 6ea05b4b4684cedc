// nectb_selftest_bounded_wait: exercises the bounded mbarrier wait of the
// tensor-core kernels on a barrier that nothing arrives at, so a test can see
// a wait run out and end with a status word instead of a hang or a fault.
#include "common.cuh"
#include "tcgen05.cuh"

namespace nectb {
namespace {

__global__ void bounded_wait_kernel(unsigned int* error_word, uint32_t max_tries) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  __syncthreads();
  // phase 0 never completes: no thread arrives on the barrier
  const bool ok = tc::mbar_wait(&bar, 0, max_tries);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) *error_word = 1u;
  else if (threadIdx.x == 0) *error_word = 0u;
}

}  // namespace
}  // namespace nectb

extern "C" int nectb_selftest_bounded_wait(unsigned int* error_word, uint32_t max_tries, void* stream) {
  using namespace nectb;
  clear_error();
  NECTB_REQUIRE(error_word, "null error word");
  NECTB_REQUIRE(max_tries > 0 && max_tries <= (1u << 16), "max_tries must be in [1, 65536]");
  bounded_wait_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(error_word, max_tries);
  return launch_status("bounded_wait_kernel");
}
