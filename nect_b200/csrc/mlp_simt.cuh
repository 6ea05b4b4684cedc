// fp32 SIMT pieces of the bias-free MLP (tiny-cuda-nn FullyFusedMLP
// semantics, as configured by MLPNetConfig in nect/config.py:115-135).
//
// Each thread owns one sample.  Its activation vectors live in shared memory
// as column t of [features][NT] arrays (thread t touches only its column, so
// per-sample work needs no barriers and accesses are bank-conflict free).
// Layer products run over 32-output groups: 32 accumulators in registers, the
// input element from the thread's column, the weight row as broadcast float4
// loads.  Loops over groups are not unrolled, which keeps the code small.
#pragma once
#include <cuda_runtime.h>

#include "../../include/nectb.h"

namespace nectb {

constexpr int kWidth = 64;

__device__ __forceinline__ float act_fwd(float z, int kind) {
  switch (kind) {
    case NECTB_ACT_RELU:
      return z > 0.f ? z : 0.f;
    case NECTB_ACT_LEAKY_RELU:
      return z > 0.f ? z : 0.01f * z;
    case NECTB_ACT_SOFTPLUS:
      return z > 20.f ? z : log1pf(expf(z));
    case NECTB_ACT_SIGMOID:
      return 1.f / (1.f + expf(-z));
    default:
      return z;
  }
}

// Derivative given the pre-activation z.
__device__ __forceinline__ float act_grad_z(float z, int kind) {
  switch (kind) {
    case NECTB_ACT_RELU:
      return z > 0.f ? 1.f : 0.f;
    case NECTB_ACT_LEAKY_RELU:
      return z > 0.f ? 1.f : 0.01f;
    case NECTB_ACT_SOFTPLUS:
      return z > 20.f ? 1.f : 1.f / (1.f + expf(-z));
    case NECTB_ACT_SIGMOID: {
      float s = 1.f / (1.f + expf(-z));
      return s * (1.f - s);
    }
    default:
      return 1.f;
  }
}

// Derivative of a hidden activation given its OUTPUT a (valid for none, relu
// and leaky relu, the hidden activations the fused kernels accept).
__device__ __forceinline__ float act_grad_a(float a, int kind) {
  switch (kind) {
    case NECTB_ACT_RELU:
      return a > 0.f ? 1.f : 0.f;
    case NECTB_ACT_LEAKY_RELU:
      return a > 0.f ? 1.f : 0.01f;
    default:
      return 1.f;
  }
}

// out[o*LD] = act(sum_k M[k][o] * in[k*LD]) for o < N.  M is [K][N] row-major
// (shared or global memory, rows 16-byte aligned); in/out point at this
// thread's column of [.][LD] arrays.  When N is not a multiple of 32 the last
// group of 32 outputs reads past the end of each row of M into the next row
// (or the next array: M must be followed by at least 32 - N % 32 floats) and
// stores only the outputs below N.
template <int K, int N, int LD>
__device__ __forceinline__ void gemv_cols(const float* __restrict__ M, const float* __restrict__ in,
                                          float* __restrict__ out, int act) {
  static_assert(N % 4 == 0, "rows of M must be 16-byte aligned");
  const int t = 0;
#pragma unroll 1
  for (int og = 0; og < N; og += 32) {
    float acc[32];
#pragma unroll
    for (int o = 0; o < 32; ++o) acc[o] = 0.f;
#pragma unroll 2
    for (int k = 0; k < K; ++k) {
      const float xk = in[k * LD + t];
      const float4* w = reinterpret_cast<const float4*>(M + k * N + og);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 v = w[q];
        acc[4 * q + 0] = fmaf(v.x, xk, acc[4 * q + 0]);
        acc[4 * q + 1] = fmaf(v.y, xk, acc[4 * q + 1]);
        acc[4 * q + 2] = fmaf(v.z, xk, acc[4 * q + 2]);
        acc[4 * q + 3] = fmaf(v.w, xk, acc[4 * q + 3]);
      }
    }
#pragma unroll
    for (int o = 0; o < 32; ++o)
      if (N % 32 == 0 || og + o < N) out[(og + o) * LD + t] = act_fwd(acc[o], act);
  }
}

// Last layer fused with the output product: returns sum_o w[o] * act(sum_k M[k][o] * in[k]).
template <int K, int LD>
__device__ __forceinline__ float gemv_dot(const float* __restrict__ M, const float* __restrict__ in,
                                          const float* __restrict__ w, int act) {
  float z = 0.f;
#pragma unroll 1
  for (int og = 0; og < kWidth; og += 32) {
    float acc[32];
#pragma unroll
    for (int o = 0; o < 32; ++o) acc[o] = 0.f;
#pragma unroll 2
    for (int k = 0; k < K; ++k) {
      const float xk = in[k * LD];
      const float4* m = reinterpret_cast<const float4*>(M + k * kWidth + og);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 v = m[q];
        acc[4 * q + 0] = fmaf(v.x, xk, acc[4 * q + 0]);
        acc[4 * q + 1] = fmaf(v.y, xk, acc[4 * q + 1]);
        acc[4 * q + 2] = fmaf(v.z, xk, acc[4 * q + 2]);
        acc[4 * q + 3] = fmaf(v.w, xk, acc[4 * q + 3]);
      }
    }
#pragma unroll
    for (int o = 0; o < 32; ++o) z = fmaf(w[og + o], act_fwd(acc[o], act), z);
  }
  return z;
}

// sum_k w[k] * in[k * LD]
template <int K, int LD>
__device__ __forceinline__ float dot_col(const float* __restrict__ w, const float* __restrict__ in) {
  float acc = 0.f;
#pragma unroll 8
  for (int k = 0; k < K; ++k) acc = fmaf(w[k], in[k * LD], acc);
  return acc;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

namespace detail {
template <int N>
__device__ __forceinline__ void rs_step(const float* in, float* out, int lane, int offset) {
  const bool up = (lane & offset) != 0;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const float send = up ? in[k] : in[k + N];
    const float keep = up ? in[k + N] : in[k];
    out[k] = keep + __shfl_xor_sync(0xffffffffu, send, offset);
  }
}
}  // namespace detail

// Butterfly reduce-scatter of 64 per-lane values over the warp: lane L ends
// with the warp sums of entries j0 and j0 + 1 (62 shuffles instead of 320 for
// 64 separate warp sums).
__device__ __forceinline__ void warp_reduce_scatter64(const float* v, int lane, float& s0, float& s1, int& j0) {
  float a[32], b[16], c[8], d[4], e[2];
  detail::rs_step<32>(v, a, lane, 16);
  detail::rs_step<16>(a, b, lane, 8);
  detail::rs_step<8>(b, c, lane, 4);
  detail::rs_step<4>(c, d, lane, 2);
  detail::rs_step<2>(d, e, lane, 1);
  s0 = e[0];
  s1 = e[1];
  j0 = ((lane >> 4) & 1) * 32 + ((lane >> 3) & 1) * 16 + ((lane >> 2) & 1) * 8 + ((lane >> 1) & 1) * 4 + (lane & 1) * 2;
}

// Weights of the SIMT paths: for every layer k the transposed copy WT_k
// [in][64] in shared memory (forward products) and the PyTorch layout W_k
// [64][in] (backward products; in shared memory too when there is room,
// else read from the global weight buffer through L1), then w_out [64].
constexpr int kMaxHidden = 6;
struct SimtWeights {
  const float* WT[kMaxHidden];
  const float* W[kMaxHidden];
  const float* wout;
};

template <int IN, int H, bool kBoth>
__host__ __device__ constexpr int simt_weight_floats() {
  return (kBoth ? 2 : 1) * (kWidth * IN + (H - 1) * kWidth * kWidth) + kWidth;
}

// Copies the fp32 weight buffer (PyTorch layout, nect's W0, W1.., w_out) into
// shared memory as SimtWeights; all threads of the block must call.  Without
// kBoth the PyTorch-layout pointers address the global buffer.
template <int IN, int H, bool kBoth>
__device__ __forceinline__ SimtWeights stage_weights(const float* __restrict__ W, float* smem) {
  static_assert(H >= 1 && H <= kMaxHidden, "hidden layers");
  SimtWeights sw;
  int off_g = 0, off_s = 0;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    const int K = (k == 0) ? IN : kWidth;
    float* WT = smem + off_s;
    float* Wd = kBoth ? smem + off_s + K * kWidth : nullptr;
    for (int e = threadIdx.x; e < K * kWidth; e += blockDim.x) {
      const float v = W[off_g + e];  // row j = e / K, column i = e % K
      if (kBoth) Wd[e] = v;
      WT[(e % K) * kWidth + e / K] = v;
    }
    sw.WT[k] = WT;
    sw.W[k] = kBoth ? Wd : W + off_g;
    off_g += K * kWidth;
    off_s += (kBoth ? 2 : 1) * K * kWidth;
  }
  float* wo = smem + off_s;
  for (int e = threadIdx.x; e < kWidth; e += blockDim.x) wo[e] = W[off_g + e];
  sw.wout = wo;
  for (int k = H; k < kMaxHidden; ++k) sw.WT[k] = sw.W[k] = nullptr;
  return sw;
}

// Hidden activations of the SIMT forward kernels: two [64][LD] buffers that
// consecutive layers alternate between.
template <int H>
__host__ __device__ constexpr int simt_hidden_buffers() {
  return H - 1 < 2 ? H - 1 : 2;
}

}  // namespace nectb
