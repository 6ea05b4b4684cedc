// Roofline probes: the throughput of random E-byte gathers from a buffer and
// of random E-byte fp32 reductions into a buffer.  With the buffer the size
// of a hash table (or of one scatter pass's gradient slice) and below the L2
// size, they measure the L2 roof that the encoding's corner gathers and the
// gradient scatter's reductions run against; above it, the HBM random-access
// roof.  Indices come from a per-thread linear congruential sequence spread
// over the buffer by a 32x32-bit high multiply, so every access is
// independent of the previous one and many are in flight per thread.
#include <algorithm>

#include "common.cuh"

namespace nectb {
namespace {

constexpr int kProbeThreads = 256;

__device__ __forceinline__ uint32_t probe_mix(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  return (uint32_t)x;
}

template <int E>
__device__ __forceinline__ uint32_t probe_load(const uint8_t* p) {
  if constexpr (E == 4) {
    return __ldg(reinterpret_cast<const uint32_t*>(p));
  } else if constexpr (E == 8) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
    return v.x ^ v.y;
  } else {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    return v.x ^ v.y ^ v.z ^ v.w;
  }
}

template <int E>
__global__ void __launch_bounds__(kProbeThreads) gather_probe_kernel(const uint8_t* __restrict__ buf, uint32_t n,
                                                                     int per_thread, uint32_t seed,
                                                                     unsigned int* __restrict__ sink) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint32_t h = probe_mix(tid * 0x9e3779b97f4a7c15ull + seed);
  uint32_t acc = 0;
#pragma unroll 8
  for (int i = 0; i < per_thread; ++i) {
    h = h * 1664525u + 1013904223u;
    const uint32_t e = (uint32_t)(((uint64_t)h * n) >> 32);
    acc ^= probe_load<E>(buf + (uint64_t)e * E);
  }
  if (acc == 0x5bd1e995u) sink[0] = acc;  // keeps the loads; practically never taken
}

template <int E>
__global__ void __launch_bounds__(kProbeThreads) reduce_probe_kernel(float* __restrict__ buf, uint32_t n,
                                                                     int per_thread, uint32_t seed) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint32_t h = probe_mix(tid * 0x9e3779b97f4a7c15ull + seed);
  const float v = 1e-30f;
#pragma unroll 8
  for (int i = 0; i < per_thread; ++i) {
    h = h * 1664525u + 1013904223u;
    const uint32_t e = (uint32_t)(((uint64_t)h * n) >> 32);
    float* dst = buf + (uint64_t)e * (E / 4);
    if constexpr (E == 4)
      atomicAdd(dst, v);
    else if constexpr (E == 8)
      atomicAdd(reinterpret_cast<float2*>(dst), make_float2(v, v));
    else
      atomicAdd(reinterpret_cast<float4*>(dst), make_float4(v, v, v, v));
  }
}

int probe_grid(int64_t n_ops, int* blocks, int* per_thread) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t threads = (int64_t)sms * 8 * kProbeThreads;  // 64 warps per SM
  *blocks = sms * 8;
  *per_thread = (int)std::max<int64_t>(1, ceil_div(n_ops, threads));
  return NECTB_OK;
}

}  // namespace
}  // namespace nectb

using namespace nectb;

extern "C" int nectb_probe_gather(const void* buf, int64_t n_entries, int32_t entry_bytes, int64_t n_gathers,
                                  unsigned int* sink, void* stream) {
  clear_error();
  NECTB_REQUIRE(buf && sink, "null buffer");
  NECTB_REQUIRE(n_entries >= 1 && n_entries <= 0xffffffffll, "n_entries must be 1..2^32-1");
  NECTB_REQUIRE(entry_bytes == 4 || entry_bytes == 8 || entry_bytes == 16, "entry_bytes must be 4, 8 or 16");
  NECTB_REQUIRE(((uintptr_t)buf % entry_bytes) == 0, "buffer not aligned to the entry size");
  NECTB_REQUIRE(n_gathers >= 1, "n_gathers must be positive");
  int blocks, per;
  probe_grid(n_gathers, &blocks, &per);
  cudaStream_t s = (cudaStream_t)stream;
  const uint8_t* b = (const uint8_t*)buf;
  const uint32_t n = (uint32_t)n_entries;
  if (entry_bytes == 4)
    gather_probe_kernel<4><<<blocks, kProbeThreads, 0, s>>>(b, n, per, 12345u, sink);
  else if (entry_bytes == 8)
    gather_probe_kernel<8><<<blocks, kProbeThreads, 0, s>>>(b, n, per, 12345u, sink);
  else
    gather_probe_kernel<16><<<blocks, kProbeThreads, 0, s>>>(b, n, per, 12345u, sink);
  return launch_status("gather_probe_kernel");
}

extern "C" int nectb_probe_reduce(float* buf, int64_t n_entries, int32_t entry_bytes, int64_t n_reductions,
                                  void* stream) {
  clear_error();
  NECTB_REQUIRE(buf, "null buffer");
  NECTB_REQUIRE(n_entries >= 1 && n_entries <= 0xffffffffll, "n_entries must be 1..2^32-1");
  NECTB_REQUIRE(entry_bytes == 4 || entry_bytes == 8 || entry_bytes == 16, "entry_bytes must be 4, 8 or 16");
  NECTB_REQUIRE(((uintptr_t)buf % entry_bytes) == 0, "buffer not aligned to the entry size");
  NECTB_REQUIRE(n_reductions >= 1, "n_reductions must be positive");
  int blocks, per;
  probe_grid(n_reductions, &blocks, &per);
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t n = (uint32_t)n_entries;
  if (entry_bytes == 4)
    reduce_probe_kernel<4><<<blocks, kProbeThreads, 0, s>>>(buf, n, per, 777u);
  else if (entry_bytes == 8)
    reduce_probe_kernel<8><<<blocks, kProbeThreads, 0, s>>>(buf, n, per, 777u);
  else
    reduce_probe_kernel<16><<<blocks, kProbeThreads, 0, s>>>(buf, n, per, 777u);
  return launch_status("reduce_probe_kernel");
}

extern "C" int64_t nectb_probe_ops(int64_t n_ops) {
  int blocks, per;
  probe_grid(n_ops, &blocks, &per);
  return (int64_t)blocks * kProbeThreads * per;
}
