// Roofline probes: the throughput of random E-byte gathers from a buffer and
// of random E-byte fp32 reductions into a buffer.  With the buffer the size
// of a hash table (or of one scatter pass's gradient slice) and below the L2
// size, they measure the L2 roof that the encoding's corner gathers and the
// gradient scatter's reductions run against; above it, the HBM random-access
// roof.  Mode 0: every lane accesses its own random entry (the access pattern
// of hashed corners); mode 1: the 32 lanes of a warp access 32 consecutive
// entries at a random warp-aligned place (whole lines: the L2's byte
// bandwidth).  Indices come from a linear congruential sequence per thread
// (mode 0) or per warp (mode 1) spread over the buffer by a 32x32-bit high
// multiply, so every access is independent of the previous one and many are
// in flight per thread.
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
  } else if constexpr (E == 16) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    return v.x ^ v.y ^ v.z ^ v.w;
  } else {  // one whole 32-byte sector
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    const uint4 b = __ldg(reinterpret_cast<const uint4*>(p + 16));
    return a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w;
  }
}

// Entry of access i: mode 0 a random entry per lane; mode 1 entry lane of a
// random group of 32 (n counts groups then).
template <int MODE>
__device__ __forceinline__ uint64_t probe_entry(uint32_t& h, uint32_t n) {
  h = h * 1664525u + 1013904223u;
  const uint64_t e = ((uint64_t)h * n) >> 32;
  return MODE == 0 ? e : e * 32 + (threadIdx.x & 31);
}

__device__ __forceinline__ uint32_t probe_seed(int mode, uint32_t seed) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  return probe_mix((mode == 0 ? tid : tid >> 5) * 0x9e3779b97f4a7c15ull + seed);
}

template <int E, int MODE>
__global__ void __launch_bounds__(kProbeThreads) gather_probe_kernel(const uint8_t* __restrict__ buf, uint32_t n,
                                                                     int per_thread, uint32_t seed,
                                                                     unsigned int* __restrict__ sink) {
  uint32_t h = probe_seed(MODE, seed);
  uint32_t acc = 0;
#pragma unroll 8
  for (int i = 0; i < per_thread; ++i) acc ^= probe_load<E>(buf + probe_entry<MODE>(h, n) * E);
  if (acc == 0x5bd1e995u) sink[0] = acc;  // keeps the loads; practically never taken
}

template <int E, int MODE>
__global__ void __launch_bounds__(kProbeThreads) reduce_probe_kernel(float* __restrict__ buf, uint32_t n,
                                                                     int per_thread, uint32_t seed) {
  uint32_t h = probe_seed(MODE, seed);
  const float v = 1e-30f;
#pragma unroll 8
  for (int i = 0; i < per_thread; ++i) {
    float* dst = buf + probe_entry<MODE>(h, n) * (E / 4);
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

extern "C" int nectb_probe_gather(const void* buf, int64_t n_entries, int32_t entry_bytes, int32_t mode,
                                  int64_t n_gathers, unsigned int* sink, void* stream) {
  clear_error();
  NECTB_REQUIRE(buf && sink, "null buffer");
  NECTB_REQUIRE(mode == 0 || mode == 1, "mode must be 0 (random entries) or 1 (random lines)");
  NECTB_REQUIRE(entry_bytes == 4 || entry_bytes == 8 || entry_bytes == 16 || entry_bytes == 32,
                "entry_bytes must be 4, 8, 16 or 32");
  const int64_t units = mode ? n_entries / 32 : n_entries;
  NECTB_REQUIRE(units >= 1 && units <= 0xffffffffll, "n_entries must give 1..2^32-1 units");
  NECTB_REQUIRE(((uintptr_t)buf % entry_bytes) == 0, "buffer not aligned to the entry size");
  NECTB_REQUIRE(n_gathers >= 1, "n_gathers must be positive");
  int blocks, per;
  probe_grid(n_gathers, &blocks, &per);
  cudaStream_t s = (cudaStream_t)stream;
  const uint8_t* b = (const uint8_t*)buf;
  const uint32_t n = (uint32_t)units;
#define NECTB_GPROBE(E)                                                                       \
  (mode ? gather_probe_kernel<E, 1><<<blocks, kProbeThreads, 0, s>>>(b, n, per, 12345u, sink) \
        : gather_probe_kernel<E, 0><<<blocks, kProbeThreads, 0, s>>>(b, n, per, 12345u, sink))
  if (entry_bytes == 4)
    NECTB_GPROBE(4);
  else if (entry_bytes == 8)
    NECTB_GPROBE(8);
  else if (entry_bytes == 16)
    NECTB_GPROBE(16);
  else
    NECTB_GPROBE(32);
#undef NECTB_GPROBE
  return launch_status("gather_probe_kernel");
}

extern "C" int nectb_probe_reduce(float* buf, int64_t n_entries, int32_t entry_bytes, int32_t mode,
                                  int64_t n_reductions, void* stream) {
  clear_error();
  NECTB_REQUIRE(buf, "null buffer");
  NECTB_REQUIRE(mode == 0 || mode == 1, "mode must be 0 (random entries) or 1 (random lines)");
  NECTB_REQUIRE(entry_bytes == 4 || entry_bytes == 8 || entry_bytes == 16, "entry_bytes must be 4, 8 or 16");
  const int64_t units = mode ? n_entries / 32 : n_entries;
  NECTB_REQUIRE(units >= 1 && units <= 0xffffffffll, "n_entries must give 1..2^32-1 units");
  NECTB_REQUIRE(((uintptr_t)buf % entry_bytes) == 0, "buffer not aligned to the entry size");
  NECTB_REQUIRE(n_reductions >= 1, "n_reductions must be positive");
  int blocks, per;
  probe_grid(n_reductions, &blocks, &per);
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t n = (uint32_t)units;
#define NECTB_RPROBE(E)                                                                   \
  (mode ? reduce_probe_kernel<E, 1><<<blocks, kProbeThreads, 0, s>>>(buf, n, per, 777u) \
        : reduce_probe_kernel<E, 0><<<blocks, kProbeThreads, 0, s>>>(buf, n, per, 777u))
  if (entry_bytes == 4)
    NECTB_RPROBE(4);
  else if (entry_bytes == 8)
    NECTB_RPROBE(8);
  else
    NECTB_RPROBE(16);
#undef NECTB_RPROBE
  return launch_status("reduce_probe_kernel");
}

extern "C" int64_t nectb_probe_ops(int64_t n_ops) {
  int blocks, per;
  probe_grid(n_ops, &blocks, &per);
  return (int64_t)blocks * kProbeThreads * per;
}
