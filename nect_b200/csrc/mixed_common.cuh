// Pieces shared by the tensor-core (tcgen05) kernels of training and
// queries: the swizzled operand tiles, the staging of the weights as bf16
// tiles, the encoder's row writer and the hidden activations.
//
// The MLP input row of L levels x F features holds IN = L * F values padded
// with zeros to INP (a multiple of the MMA's K step of 16), split over KT
// tiles of 64 columns (InShape in common.cuh).  Weight tiles: W0 as KT tiles
// [64 outputs][64 inputs], then one [64][64] tile per further hidden layer;
// w_out stays fp32.
#pragma once
#include <cuda_fp16.h>

#include "common.cuh"
#include "hashgrid.cuh"
#include "mlp_simt.cuh"
#include "tcgen05.cuh"

namespace nectb {

constexpr uint32_t kTile = 128 * 128;  // bytes of a [128][64 bf16] tile
constexpr uint32_t kWTile = 64 * 128;  // bytes of a [64][64 bf16] tile

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// fp32 weights (PyTorch layout) -> bf16 swizzled tiles: W0 rows o over KT
// tiles (input columns beyond IN are zero), W1..W_{H-1} rows o in the tiles
// after them; w_out fp32.
template <int L, int F, int H>
__device__ __forceinline__ void stage_mixed_weights(const float* __restrict__ W, uint8_t* sW, float* sWout) {
  using S = InShape<L, F>;
  constexpr int IN = S::IN;
  for (int e = threadIdx.x; e < 64 * S::KT * 8; e += blockDim.x) {
    const int o = e / (S::KT * 8), j = e % (S::KT * 8);
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = (8 * j + q < IN) ? W[o * IN + 8 * j + q] : 0.f;
    tc::st_chunk_bf16(sW + (j / 8) * kWTile, o, j % 8, v);
  }
#pragma unroll 1
  for (int k = 1; k < H; ++k) {
    const float* Wk = W + 64 * IN + (k - 1) * 64 * 64;
    for (int e = threadIdx.x; e < 64 * 8; e += blockDim.x) {
      const int o = e / 8, j = e % 8;
      float v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = Wk[o * 64 + 8 * j + q];
      tc::st_chunk_bf16(sW + (S::KT + k - 1) * kWTile, o, j, v);
    }
  }
  for (int e = threadIdx.x; e < 64; e += blockDim.x) sWout[e] = W[64 * IN + (H - 1) * 64 * 64 + e];
}

// Hidden activation of the tensor-core paths (ReLU, LeakyReLU or none; the
// shapes validate_mlp accepts) and its derivative from the sign of the
// pre-activation.
__device__ __forceinline__ float hidden_act(float x, int act) {
  return act == NECTB_ACT_RELU ? fmaxf(x, 0.f) : (act == NECTB_ACT_LEAKY_RELU ? (x > 0.f ? x : 0.01f * x) : x);
}
// g times the activation's slope at a pre-activation of the given sign.
__device__ __forceinline__ float hidden_grad(float g, bool positive, int act) {
  return act == NECTB_ACT_RELU ? (positive ? g : 0.f) : (act == NECTB_ACT_LEAKY_RELU ? (positive ? g : 0.01f * g) : g);
}

// Activation of 64 accumulator values into row r of a bf16 tile; bit j of m = (x_j > 0).
__device__ __forceinline__ void act_row(const float* h, uint8_t* tile, int r, int act, uint32_t& mlo, uint32_t& mhi) {
  mlo = 0;
  mhi = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float x = h[8 * j + q];
      v[q] = hidden_act(x, act);
      const uint32_t bit = x > 0.f ? 1u : 0u;
      if (8 * j + q < 32) mlo |= bit << (8 * j + q); else mhi |= bit << (8 * j + q - 32);
    }
    tc::st_chunk_bf16(tile, r, j, v);
  }
}

// Encodes one sample into row r of the swizzled X tiles (bf16), 8 features
// (one 16-byte chunk) at a time, the padding after the last level zero;
// invalid samples write zeros.  With xdst the row is also written there
// (evict-first: the store streams past the L2 that holds the tables).
template <int D, int F, int L>
__device__ __forceinline__ void encode_row(const GridDev& g, const __half* __restrict__ table, const float* p,
                                           bool valid, uint8_t* sX, int r, uint4* __restrict__ xdst = nullptr) {
  using S = InShape<L, F>;
  constexpr int LPC = 8 / F;  // levels per 16-byte chunk
#pragma unroll 1
  for (int j = 0; j < S::NCH; ++j) {
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = 0.f;
    if (valid) {
#pragma unroll
      for (int q = 0; q < LPC; ++q) {
        const int l = j * LPC + q;
        if (L % LPC != 0 && l >= L) break;   // the padding chunk after an odd last level
        LevelCorners<D> lc;
        level_corners<D>(g, l, p, lc);
        float vals[1 << D][F];
        // the odd hashed levels' corners through the texture path (a second
        // L1 data pipe beside the load/store unit's), the others as loads
        if (g.tex && ((g.hashed_bits >> l) & 1u) && (l & 1)) {
#pragma unroll
          for (int c = 0; c < (1 << D); ++c) {
            const int e = (int)(g.offset[l] + lc.idx[c]);
            if constexpr (F == 2) {
              const unsigned int raw = tex1Dfetch<unsigned int>((cudaTextureObject_t)g.tex, e);
              const float2 v = __half22float2(*reinterpret_cast<const __half2*>(&raw));
              vals[c][0] = v.x;
              vals[c][1] = v.y;
            } else {
              const uint2 raw = tex1Dfetch<uint2>((cudaTextureObject_t)g.tex, e);
              const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
              const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
              vals[c][0] = a.x;
              vals[c][1] = a.y;
              vals[c][2] = b.x;
              vals[c][3] = b.y;
            }
          }
        } else
#pragma unroll
        for (int c = 0; c < (1 << D); ++c) Feat<F, __half>::load(table, g.offset[l] + lc.idx[c], vals[c]);
#pragma unroll
        for (int f = 0; f < F; ++f) {
          float acc = 0.f;
#pragma unroll
          for (int c = 0; c < (1 << D); ++c) acc = fmaf(lc.w[c], vals[c][f], acc);
          v[q * F + f] = acc;
        }
      }
    }
    const uint4 packed = tc::pack_bf16x8(v);
    tc::st_chunk_raw(sX + (j / 8) * kTile, r, j % 8, packed);
    if (xdst) __stcs(xdst + j, packed);
  }
}

// Loads 64 fp32 TMEM columns [col, col+64) of this thread's lane.
__device__ __forceinline__ void ld64(uint32_t taddr, float* v) {
#pragma unroll
  for (int c = 0; c < 4; ++c) tc::tmem_ld16(taddr + 16 * c, v + 16 * c);
  tc::tmem_wait_ld();
}

}  // namespace nectb
