// Multiresolution hash encoding on the device: per-level layout, corner
// indices and weights, gather (forward) and atomic scatter (backward).
//
// Method: Mueller et al., "Instant Neural Graphics Primitives with a
// Multiresolution Hash Encoding", ACM TOG 41(4), 2022, section 3 (the
// encoding the reference takes from tiny-cuda-nn, nect/network/networks.py:
// 52-57 and 478-481).  Build-defined details, identical in oracle/hashgrid.py:
//   - level resolution floor(base * scale^l) (t axis: floor(base_t * scale^l));
//   - p = x * res in fp32, cell = clamp(floor(p), 0, res-1), frac = p - cell;
//   - dense storage when (res+1)^d vertices fit in T (entries rounded up to a
//     multiple of 8), else hash XOR_k v_k * pi_k mod T with
//     pi = (1, 2654435761, 805459861, 2246822519);
//   - axis k of the input (z, y, x[, t]) has pi_k / stride_k.
// Corner c has bit k set when it takes the upper vertex along axis k; its
// weight is the product over k of (bit ? frac_k : 1 - frac_k) in axis order.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>

#include "../../include/nectb.h"

namespace nectb {

constexpr uint32_t kPrime1 = 2654435761u;
constexpr uint32_t kPrime2 = 805459861u;
constexpr uint32_t kPrime3 = 2246822519u;

struct GridDev {
  int n_dims;
  int n_levels;
  int n_features;
  uint32_t hash_mask;
  uint32_t hashed_bits;  // bit l: level l is hashed
  int res[NECTB_MAX_LEVELS][4];
  uint32_t stride[NECTB_MAX_LEVELS][4];
  int64_t offset[NECTB_MAX_LEVELS];  // first entry of level l
  int64_t total_entries;
  unsigned long long tex = 0;        // texture object over an fp16 table (0: none)
};

// Host: fill GridDev from the C-ABI description (returns false when invalid).
bool make_grid_dev(const NectbHashGrid* g, GridDev* out);

template <int D>
struct LevelCorners {
  uint32_t idx[1 << D];  // entry index within the level
  float w[1 << D];
  uint64_t cell;         // spatial cell (z, y, x) packed 21 bits per axis
};

template <int D>
__device__ __forceinline__ void level_corners(const GridDev& g, int l, const float* x, LevelCorners<D>& lc) {
  int c[D];
  float f[D];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const int r = g.res[l][k];
    // p is the fp32-rounded product for the floor and the fraction alike:
    // __fmul_rn keeps the compiler from contracting p - ci into an fma, which
    // would give the unrounded product's fraction in some kernels only
    const float p = __fmul_rn(x[k], (float)r);
    int ci = (int)floorf(p);
    ci = ci < 0 ? 0 : (ci > r - 1 ? r - 1 : ci);
    c[k] = ci;
    f[k] = p - (float)ci;
  }
  lc.cell = (uint64_t)(uint32_t)c[0] | ((uint64_t)(uint32_t)c[1] << 21) | ((uint64_t)(uint32_t)c[2] << 42);
  const bool hashed = (g.hashed_bits >> l) & 1u;
  // Per-axis terms of the lower/upper vertex: the hash XORs v_k * pi_k and the
  // dense index adds v_k * stride_k, and (c+1)*m = c*m + m in 32-bit
  // arithmetic, so each corner costs one XOR/add per axis.  Identical integers
  // to evaluating every corner from scratch.
  uint32_t term[D][2];
  float wt[D][2];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    uint32_t m;
    if (hashed)
      m = (k == 0) ? 1u : (k == 1 ? kPrime1 : (k == 2 ? kPrime2 : kPrime3));
    else
      m = (k == 0) ? 1u : g.stride[l][k];
    term[k][0] = (uint32_t)c[k] * m;
    term[k][1] = term[k][0] + m;
    wt[k][0] = 1.f - f[k];
    wt[k][1] = f[k];
  }
  // Weight products in axis order, shared prefixes computed once.
  float w01[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) w01[q] = wt[0][q & 1] * wt[1][(q >> 1) & 1];
#pragma unroll
  for (int corner = 0; corner < (1 << D); ++corner) {
    uint32_t id = term[0][corner & 1];
#pragma unroll
    for (int k = 1; k < D; ++k) id = hashed ? (id ^ term[k][(corner >> k) & 1]) : (id + term[k][(corner >> k) & 1]);
    if (hashed) id &= g.hash_mask;
    float w = w01[corner & 3];
#pragma unroll
    for (int k = 2; k < D; ++k) w = w * wt[k][(corner >> k) & 1];
    lc.idx[corner] = id;
    lc.w[corner] = w;
  }
}

// ---- feature loads -----------------------------------------------------
template <int F, typename T>
struct Feat;

template <>
struct Feat<2, float> {
  static __device__ __forceinline__ void load(const float* base, int64_t entry, float* out) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(base + entry * 2));
    out[0] = v.x;
    out[1] = v.y;
  }
};
template <>
struct Feat<4, float> {
  static __device__ __forceinline__ void load(const float* base, int64_t entry, float* out) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(base + entry * 4));
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
  }
};
template <>
struct Feat<2, __half> {
  static __device__ __forceinline__ void load(const __half* base, int64_t entry, float* out) {
    const unsigned int raw = __ldg(reinterpret_cast<const unsigned int*>(base + entry * 2));
    const __half2 h = *reinterpret_cast<const __half2*>(&raw);
    const float2 v = __half22float2(h);
    out[0] = v.x;
    out[1] = v.y;
  }
};
template <>
struct Feat<4, __half> {
  static __device__ __forceinline__ void load(const __half* base, int64_t entry, float* out) {
    const uint2 raw = __ldg(reinterpret_cast<const uint2*>(base + entry * 4));
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
    out[0] = a.x;
    out[1] = a.y;
    out[2] = b.x;
    out[3] = b.y;
  }
};

// Encodes one point: out[(l*F + f) * stride] for all levels.  x has D
// coordinates in [0,1].
template <int D, int F, typename T>
__device__ __forceinline__ void encode_point(const GridDev& g, const T* __restrict__ table, const float* x,
                                             float* out, int stride = 1) {
#pragma unroll 1
  for (int l = 0; l < g.n_levels; ++l) {
    LevelCorners<D> lc;
    level_corners<D>(g, l, x, lc);
    float vals[1 << D][F];
#pragma unroll
    for (int c = 0; c < (1 << D); ++c) Feat<F, T>::load(table, g.offset[l] + lc.idx[c], vals[c]);
    float acc[F];
#pragma unroll
    for (int f = 0; f < F; ++f) acc[f] = 0.f;
#pragma unroll
    for (int c = 0; c < (1 << D); ++c)
#pragma unroll
      for (int f = 0; f < F; ++f) acc[f] = fmaf(lc.w[c], vals[c][f], acc[f]);
#pragma unroll
    for (int f = 0; f < F; ++f) out[(l * F + f) * stride] = acc[f];
  }
}

// Gradient scatter of one point: grad[offset + idx][f] += w * dout[(l*F + f) * stride].
template <int D, int F>
__device__ __forceinline__ void scatter_point(const GridDev& g, float* __restrict__ grad, const float* x,
                                              const float* dsrc, int stride = 1) {
#pragma unroll 1
  for (int l = 0; l < g.n_levels; ++l) {
    LevelCorners<D> lc;
    level_corners<D>(g, l, x, lc);
    float d[F];
#pragma unroll
    for (int f = 0; f < F; ++f) d[f] = dsrc[(l * F + f) * stride];
#pragma unroll
    for (int c = 0; c < (1 << D); ++c) {
      float* dst = grad + (g.offset[l] + lc.idx[c]) * F;
      if constexpr (F == 2) {
        atomicAdd(reinterpret_cast<float2*>(dst), make_float2(lc.w[c] * d[0], lc.w[c] * d[1]));
      } else if constexpr (F == 4) {
        atomicAdd(reinterpret_cast<float4*>(dst),
                  make_float4(lc.w[c] * d[0], lc.w[c] * d[1], lc.w[c] * d[2], lc.w[c] * d[3]));
      } else {
#pragma unroll
        for (int f = 0; f < F; ++f) atomicAdd(dst + f, lc.w[c] * d[f]);
      }
    }
  }
}

// Levels on which the 32 consecutive samples a warp holds of one ray share
// cells: expected samples per cell = 1 / (res * (|dx| + |dy| + |dz|)) in
// normalised coordinates.  Bit l is set when res * (|dx| + |dy| + |dz|) is
// below the threshold.  Defaults (NectbTuning): 1.0 (3D) and 3.0 (4D, where
// merging a run costs half the shuffles: separable time weights), the values
// the autotuner picked on the 512^2 cone workloads.
__device__ __forceinline__ uint32_t run_levels(const GridDev& g, double dx, double dy, double dz, float threshold) {
  const float cross = (float)(fabs(dx) + fabs(dy) + fabs(dz));
  uint32_t m = 0;
  for (int l = 0; l < g.n_levels; ++l)
    if ((float)g.res[l][0] * cross < threshold) m |= 1u << l;
  return m;
}

// Adds the contributions of corners c and c + 1 (which differ along axis 0,
// the axis with hash prime 1 and dense stride 1): when their entries form an
// aligned pair (i0 even and i1 = i0 + 1, or i1 even and i0 = i1 + 1: on a
// hashed level with an even cell coordinate the two entries differ in the
// lowest bit only, in either order) one 16-byte reduction carries both,
// otherwise one 8-byte reduction each.  The gradient table must be 16-byte
// aligned (level offsets are multiples of 8 entries).
__device__ __forceinline__ void red_pair_f2(float* base, uint32_t i0, uint32_t i1, float a0, float a1, float b0,
                                            float b1) {
  float* dst = base + (int64_t)i0 * 2;
  if (!(i0 & 1u) && i1 == i0 + 1u) {
    atomicAdd(reinterpret_cast<float4*>(dst), make_float4(a0, a1, b0, b1));
  } else if (!(i1 & 1u) && i0 == i1 + 1u) {
    atomicAdd(reinterpret_cast<float4*>(base + (int64_t)i1 * 2), make_float4(b0, b1, a0, a1));
  } else {
    atomicAdd(reinterpret_cast<float2*>(dst), make_float2(a0, a1));
    atomicAdd(reinterpret_cast<float2*>(base + (int64_t)i1 * 2), make_float2(b0, b1));
  }
}

template <int F>
__device__ __forceinline__ void red_entry(float* dst, const float* v) {
  if constexpr (F == 2) atomicAdd(reinterpret_cast<float2*>(dst), make_float2(v[0], v[1]));
  else if constexpr (F == 4) atomicAdd(reinterpret_cast<float4*>(dst), make_float4(v[0], v[1], v[2], v[3]));
  else
#pragma unroll
    for (int f = 0; f < F; ++f) atomicAdd(dst + f, v[f]);
}

// fp32 value of a gradient element held as fp32 or bf16.
__device__ __forceinline__ float grad_value(float v) { return v; }
__device__ __forceinline__ float grad_value(__nv_bfloat16 v) { return __bfloat162float(v); }

// F consecutive gradient elements (fp32 or bf16) as one vector load; src is
// aligned to F elements.
template <int F, typename S>
__device__ __forceinline__ void load_grad_row(const S* src, float* d) {
  static_assert(F == 2 || F == 4, "F must be 2 or 4");
  if constexpr (sizeof(S) == 4 && F == 4) {
    const float4 v = *reinterpret_cast<const float4*>(src);
    d[0] = v.x, d[1] = v.y, d[2] = v.z, d[3] = v.w;
  } else if constexpr (sizeof(S) == 4) {
    const float2 v = *reinterpret_cast<const float2*>(src);
    d[0] = v.x, d[1] = v.y;
  } else if constexpr (F == 4) {
    const uint2 raw = *reinterpret_cast<const uint2*>(src);
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
    d[0] = a.x, d[1] = a.y, d[2] = b.x, d[3] = b.y;
  } else {
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(src));
    d[0] = a.x, d[1] = a.y;
  }
}

// Sum of v over the lanes [lane, end] of the lane's run (lanes after it in the
// same run); valid in the run's first lane.
__device__ __forceinline__ float run_sum(float v, int lane, int end) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float tv = __shfl_down_sync(0xffffffffu, v, o);
    if (lane + o <= end) v += tv;
  }
  return v;
}

// Warp-cooperative gradient scatter of 32 samples of one ray (all lanes call;
// `valid` masks lanes without a sample).  On levels in agg_levels, lanes in the
// same cell form contiguous runs along the ray; each run's contributions to
// each corner are summed with a segmented shuffle reduction and written by the
// run's first lane, so the table sees one atomic per (cell, corner) instead of
// one per sample.  In 4D the time weight is the same for every sample of a
// batch, so runs sum the 8 spatial corners and scale by the two time weights.
// Other levels scatter per sample.  Sums equal the per-sample atomics up to
// fp32 reassociation.
//
// dL/d(feature f of level l) is read at dsrc[l * lstride + f * fstride] (fp32,
// or bf16 with S = __nv_bfloat16); only levels [l0, l1) are scattered.  kStreamSrc: dsrc is global memory read once
// (the staging buffer, fstride 1, rows aligned to F floats): one vector load
// per level, evict-first, so the streamed rows do not push the gradient slice
// out of L2.
//
// kAdaptive: agg_levels is ignored; every level merges runs when the warp's
// 32 points form at most 24 runs of equal cells (points in no known order,
// such as a module's batch).
//
// kVecSrc: fstride is 1 and each level's F elements are one aligned vector
// (load_grad_row).
template <int D, int F, bool kStreamSrc = false, bool kAdaptive = false, typename S = float, bool kVecSrc = false>
__device__ __forceinline__ void scatter_warp(const GridDev& g, float* __restrict__ grad, const float* x, bool valid,
                                             const S* dsrc, int64_t lstride, int fstride, uint32_t agg_levels,
                                             int l0, int l1) {
  static_assert(!kStreamSrc || sizeof(S) == 4, "the streamed source is fp32");
  const int lane = threadIdx.x & 31;
#pragma unroll 1
  for (int l = l0; l < l1; ++l) {
    LevelCorners<D> lc;
    level_corners<D>(g, l, x, lc);
    float d[F];
    if constexpr (kStreamSrc && F == 2) {
      const float2 v = valid ? __ldcs(reinterpret_cast<const float2*>(dsrc + l * lstride)) : make_float2(0.f, 0.f);
      d[0] = v.x;
      d[1] = v.y;
    } else if constexpr (kStreamSrc && F == 4) {
      const float4 v =
          valid ? __ldcs(reinterpret_cast<const float4*>(dsrc + l * lstride)) : make_float4(0.f, 0.f, 0.f, 0.f);
      d[0] = v.x;
      d[1] = v.y;
      d[2] = v.z;
      d[3] = v.w;
    } else if constexpr (kVecSrc) {
      if (valid) {
        load_grad_row<F, S>(dsrc + l * lstride, d);
      } else {
#pragma unroll
        for (int f = 0; f < F; ++f) d[f] = 0.f;
      }
    } else {
#pragma unroll
      for (int f = 0; f < F; ++f) d[f] = valid ? grad_value(dsrc[l * lstride + f * fstride]) : 0.f;
    }
    float* base = grad + g.offset[l] * F;
    bool merge = kAdaptive || ((agg_levels >> l) & 1u);
    bool head = false;
    uint32_t heads = 0;
    if (merge) {
      // runs of lanes in the same spatial cell (t is the same for the whole
      // batch, so the spatial cell fixes every corner index)
      const uint64_t key = valid ? lc.cell : ~uint64_t(0);
      const uint64_t prev = __shfl_up_sync(0xffffffffu, key, 1);
      head = (lane == 0) || (prev != key);
      heads = __ballot_sync(0xffffffffu, head);
      if constexpr (kAdaptive) merge = __popc(heads) <= 24;
    }
    if (merge) {
      const uint32_t later = heads & ~((2u << lane) - 1u);
      const int end = later ? (__ffs(later) - 2) : 31;
      constexpr int SC = D == 4 ? 8 : (1 << D);   // corners summed along the run
      float ws[SC];
      float wt0 = 1.f, wt1 = 1.f;
      if constexpr (D == 4) {
        LevelCorners<3> ls;   // spatial weights (the 4D weights are these times the time weight)
        level_corners<3>(g, l, x, ls);
#pragma unroll
        for (int c = 0; c < 8; ++c) ws[c] = ls.w[c];
        const int r = g.res[l][3];
        const float pt = __fmul_rn(x[3], (float)r);   // as level_corners
        int ct = (int)floorf(pt);
        ct = ct < 0 ? 0 : (ct > r - 1 ? r - 1 : ct);
        wt1 = pt - (float)ct;
        wt0 = 1.f - wt1;
      } else {
#pragma unroll
        for (int c = 0; c < SC; ++c) ws[c] = lc.w[c];
      }
#pragma unroll
      for (int c = 0; c < SC; c += 2) {
        float s0[F], s1[F];
#pragma unroll
        for (int f = 0; f < F; ++f) {
          s0[f] = run_sum(ws[c] * d[f], lane, end);
          s1[f] = run_sum(ws[c + 1] * d[f], lane, end);
        }
        if (head && valid) {
#pragma unroll
          for (int tb = 0; tb < (D == 4 ? 2 : 1); ++tb) {
            const float wt = D == 4 ? (tb ? wt1 : wt0) : 1.f;
            const int c0 = c + tb * 8;
            if constexpr (F == 2) {
              red_pair_f2(base, lc.idx[c0], lc.idx[c0 + 1], wt * s0[0], wt * s0[1], wt * s1[0], wt * s1[1]);
            } else {
              float v0[F], v1[F];
#pragma unroll
              for (int f = 0; f < F; ++f) {
                v0[f] = wt * s0[f];
                v1[f] = wt * s1[f];
              }
              red_entry<F>(base + (int64_t)lc.idx[c0] * F, v0);
              red_entry<F>(base + (int64_t)lc.idx[c0 + 1] * F, v1);
            }
          }
        }
      }
    } else if (valid) {
#pragma unroll
      for (int c = 0; c < (1 << D); c += 2) {
        if constexpr (F == 2) {
          red_pair_f2(base, lc.idx[c], lc.idx[c + 1], lc.w[c] * d[0], lc.w[c] * d[1], lc.w[c + 1] * d[0],
                      lc.w[c + 1] * d[1]);
        } else {
          float v0[F], v1[F];
#pragma unroll
          for (int f = 0; f < F; ++f) {
            v0[f] = lc.w[c] * d[f];
            v1[f] = lc.w[c + 1] * d[f];
          }
          red_entry<F>(base + (int64_t)lc.idx[c] * F, v0);
          red_entry<F>(base + (int64_t)lc.idx[c + 1] * F, v1);
        }
      }
    }
  }
}

}  // namespace nectb
