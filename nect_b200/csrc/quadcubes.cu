// QuadCubes' composite encoding (nect/network/networks.py:392-449): four 3D
// grids of one configuration over (z, y, x), (y, x, t), (x, z, t) and
// (z, y, t) of each point, with one t for every point of a call, written as
// rows of the MLP's input matrix, and its backward.
//
// Planes.  Three of the grids have t as their last coordinate.  With t fixed,
// a level's trilinear interpolation over (a, b, t) is a bilinear
// interpolation over (a, b) of the blend w0 * v(a, b, t0) + w1 * v(a, b, t0+1)
// (weights and t0 as level_corners computes them for axis 2).  Per call and
// grid the blend is built once into a plane: a dense 2D array of the level's
// (res+1)^2 vertices where that fits in T entries, else (hashed levels) the
// T entries keyed by the (a, b) part of the hash, which is an XOR of per-axis
// terms, so v(a, b, t_v) sits at (key ^ (t_v * pi_2)) & mask.  The grids then
// gather 4 corners from a plane a few tens of MB in size (L2-resident)
// instead of 8 corners spread over a table of up to 2^23 entries per level.
// In the backward the points reduce into a plane-shaped fp32 gradient
// (L2-resident), which is spread to the two time vertices of each of its
// non-zero entries.  Results equal the 3D grid's up to fp32 reassociation
// (fp32 planes) or one fp16 rounding of the blended values (fp16 planes, the
// mixed path, whose MLP then rounds to bf16).
#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>

#include "common.cuh"
#include "hashgrid.cuh"

namespace nectb {
namespace {

struct Plane {
  int n_levels;
  uint32_t hash_mask;
  uint32_t hashed3;   // bit l: the 3D level is hashed
  uint32_t hashed2;   // bit l: the plane level keeps the T hashed entries
  int res[NECTB_MAX_LEVELS];
  int64_t stride2[NECTB_MAX_LEVELS];   // dense 3D stride of the t axis, (res+1)^2
  int64_t off3[NECTB_MAX_LEVELS];      // 3D level offsets (entries)
  int64_t off2[NECTB_MAX_LEVELS];      // plane level offsets (entries)
  int64_t n2[NECTB_MAX_LEVELS];        // plane entries that hold a value
  int64_t total2;
};

bool make_plane(const GridDev& g, Plane* p) {
  if (g.n_dims != 3) return false;
  p->n_levels = g.n_levels;
  p->hash_mask = g.hash_mask;
  p->hashed3 = g.hashed_bits;
  p->hashed2 = 0;
  const int64_t T = (int64_t)g.hash_mask + 1;
  int64_t off = 0;
  for (int l = 0; l < g.n_levels; ++l) {
    const int r = g.res[l][0];
    if (g.res[l][1] != r || g.res[l][2] != r) return false;
    const int64_t v2 = (int64_t)(r + 1) * (r + 1);
    p->res[l] = r;
    p->stride2[l] = v2;
    p->off3[l] = g.offset[l];
    p->off2[l] = off;
    if (v2 <= T) {
      p->n2[l] = v2;
    } else {
      p->n2[l] = T;
      p->hashed2 |= 1u << l;
    }
    off += (p->n2[l] + 7) / 8 * 8;
  }
  p->total2 = off;
  return true;
}

// t -> lower time vertex and its weights, as level_corners computes them.
struct TimeVertex {
  int c;
  float w0, w1;
};
__device__ __forceinline__ TimeVertex time_vertex(float t, int r) {
  const float p = __fmul_rn(t, (float)r);   // rounded product, as level_corners
  int ci = (int)floorf(p);
  ci = ci < 0 ? 0 : (ci > r - 1 ? r - 1 : ci);
  const float f = p - (float)ci;
  return {ci, 1.f - f, f};
}

// The two 3D entries (within the level) of plane entry k at time vertices
// c and c + 1.
__device__ __forceinline__ void plane_sources(const Plane& s, int l, int64_t k, int c, int64_t* e0, int64_t* e1) {
  const uint32_t tt = (uint32_t)c * kPrime2;
  if ((s.hashed2 >> l) & 1u) {
    *e0 = (int64_t)((uint64_t)k ^ (uint64_t)(tt & s.hash_mask));
    *e1 = (int64_t)((uint64_t)k ^ (uint64_t)((tt + kPrime2) & s.hash_mask));
  } else if ((s.hashed3 >> l) & 1u) {
    const uint32_t r1 = (uint32_t)s.res[l] + 1u;
    const uint32_t a = (uint32_t)(k % r1), b = (uint32_t)(k / r1);
    const uint32_t h = a ^ (b * kPrime1);
    *e0 = (int64_t)((h ^ tt) & s.hash_mask);
    *e1 = (int64_t)((h ^ (tt + kPrime2)) & s.hash_mask);
  } else {
    *e0 = k + (int64_t)c * s.stride2[l];
    *e1 = *e0 + s.stride2[l];
  }
}

template <typename T>
__device__ __forceinline__ T from_float(float v);
template <>
__device__ __forceinline__ float from_float<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half from_float<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_float<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// Stores F features (F * sizeof(O) bytes, aligned to that size) as O.
template <int F, typename O>
__device__ __forceinline__ void store_features(O* dst, const float* v) {
  if constexpr (sizeof(O) == 4 && F == 4) {
    *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
  } else if constexpr (sizeof(O) == 4 && F == 2) {
    *reinterpret_cast<float2*>(dst) = make_float2(v[0], v[1]);
  } else if constexpr (F == 4) {
    __nv_bfloat162 lo = __floats2bfloat162_rn(v[0], v[1]), hi = __floats2bfloat162_rn(v[2], v[3]);
    uint2 raw;
    raw.x = *reinterpret_cast<unsigned int*>(&lo);
    raw.y = *reinterpret_cast<unsigned int*>(&hi);
    *reinterpret_cast<uint2*>(dst) = raw;
  } else {
    *reinterpret_cast<__nv_bfloat162*>(dst) = __floats2bfloat162_rn(v[0], v[1]);
  }
}

// Builds the plane of every level (grid y = level) from the fp32 table;
// padding entries are zero.
template <int F, typename P>
__global__ void plane_build_kernel(Plane s, const float* __restrict__ table, const float* __restrict__ t,
                                   P* __restrict__ plane) {
  const int l = blockIdx.y;
  const int64_t n = (l + 1 < s.n_levels ? s.off2[l + 1] : s.total2) - s.off2[l];
  const TimeVertex tv = time_vertex(__ldg(t), s.res[l]);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    P* dst = plane + (s.off2[l] + k) * F;
    if (k >= s.n2[l]) {
#pragma unroll
      for (int f = 0; f < F; ++f) dst[f] = from_float<P>(0.f);
      continue;
    }
    int64_t e0, e1;
    plane_sources(s, l, k, tv.c, &e0, &e1);
    float a[F], b[F];
    Feat<F, float>::load(table, s.off3[l] + e0, a);
    Feat<F, float>::load(table, s.off3[l] + e1, b);
#pragma unroll
    for (int f = 0; f < F; ++f) dst[f] = from_float<P>(fmaf(tv.w0, a[f], tv.w1 * b[f]));
  }
}

// Corners of (a, b) on a plane level: entry indices (within the level) and
// bilinear weights, corner q taking the upper vertex along a when bit 0 is
// set and along b when bit 1 is set; the cell key identifies (a, b)'s cell.
struct PlaneCorners {
  uint32_t idx[4];
  float w[4];
  uint64_t cell;
};
__device__ __forceinline__ void plane_corners(const Plane& s, int l, float a, float b, PlaneCorners& pc) {
  const int r = s.res[l];
  const float pa = __fmul_rn(a, (float)r), pb = __fmul_rn(b, (float)r);   // rounded products, as level_corners
  int ia = (int)floorf(pa), ib = (int)floorf(pb);
  ia = ia < 0 ? 0 : (ia > r - 1 ? r - 1 : ia);
  ib = ib < 0 ? 0 : (ib > r - 1 ? r - 1 : ib);
  const float fa = pa - (float)ia, fb = pb - (float)ib;
  pc.cell = (uint64_t)(uint32_t)ia | ((uint64_t)(uint32_t)ib << 32);
  const bool hashed = (s.hashed2 >> l) & 1u;
  const uint32_t mb = hashed ? kPrime1 : (uint32_t)r + 1u;
  const uint32_t ta[2] = {(uint32_t)ia, (uint32_t)ia + 1u};
  const uint32_t tb[2] = {(uint32_t)ib * mb, (uint32_t)ib * mb + mb};
  const float wa[2] = {1.f - fa, fa}, wb[2] = {1.f - fb, fb};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    pc.idx[q] = hashed ? ((ta[q & 1] ^ tb[q >> 1]) & s.hash_mask) : (ta[q & 1] + tb[q >> 1]);
    pc.w[q] = wa[q & 1] * wb[q >> 1];
  }
}

// One thread per point: the plane grid's features of (zyx[ca], zyx[cb]) into
// out[i * ld + col0 + l * F + f].
template <int F, typename P, typename O>
__global__ void plane_encode_kernel(Plane s, const P* __restrict__ plane, const float* __restrict__ zyx, int64_t n,
                                    int ca, int cb, O* __restrict__ out, int64_t ld, int col0) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float a = zyx[i * 3 + ca], b = zyx[i * 3 + cb];
  O* row = out + i * ld + col0;
#pragma unroll 2   // two levels' gathers in flight
  for (int l = 0; l < s.n_levels; ++l) {
    PlaneCorners pc;
    plane_corners(s, l, a, b, pc);
    float v[4][F];
#pragma unroll
    for (int q = 0; q < 4; ++q) Feat<F, P>::load(plane, s.off2[l] + pc.idx[q], v[q]);
    float acc[F];
#pragma unroll
    for (int f = 0; f < F; ++f) {
      acc[f] = 0.f;
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[f] = fmaf(pc.w[q], v[q][f], acc[f]);
    }
    store_features<F, O>(row + l * F, acc);
  }
}

// One thread per point: the (z, y, x) grid's features into columns
// [0, L * F) of the row, the raw inputs (z, y, x, t) after the four grids when
// `identity`, and zeros from column `pad` to the end of the row.
template <int F, typename O>
__global__ void volume_encode_kernel(GridDev g, const float* __restrict__ table, const float* __restrict__ zyx,
                                     const float* __restrict__ t, int64_t n, int identity, O* __restrict__ out,
                                     int64_t ld, int pad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x[3] = {zyx[i * 3], zyx[i * 3 + 1], zyx[i * 3 + 2]};
  O* row = out + i * ld;
#pragma unroll 2   // two levels' gathers in flight
  for (int l = 0; l < g.n_levels; ++l) {
    LevelCorners<3> lc;
    level_corners<3>(g, l, x, lc);
    float v[8][F];
#pragma unroll
    for (int c = 0; c < 8; ++c) Feat<F, float>::load(table, g.offset[l] + lc.idx[c], v[c]);
    float acc[F];
#pragma unroll
    for (int f = 0; f < F; ++f) {
      acc[f] = 0.f;
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[f] = fmaf(lc.w[c], v[c][f], acc[f]);
    }
    store_features<F, O>(row + l * F, acc);
  }
  int col = 4 * g.n_levels * F;
  if (identity) {
    row[col] = from_float<O>(x[0]);
    row[col + 1] = from_float<O>(x[1]);
    row[col + 2] = from_float<O>(x[2]);
    row[col + 3] = from_float<O>(__ldg(t));
  }
  for (int c = pad; c < ld; ++c) row[c] = from_float<O>(0.f);
}

// Gradient of levels [l0, l1) of the (z, y, x) grid: dL/d(features) in
// columns [0, L * F) of the rows; warps merge runs of points in one cell
// (scatter_warp, adaptive).
template <int F, typename S>
__global__ void volume_scatter_kernel(GridDev g, const float* __restrict__ zyx, int64_t n,
                                      const S* __restrict__ dout, int64_t ld, float* __restrict__ grad, int l0,
                                      int l1) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool valid = i < n;   // every lane takes part in the warp's shuffles
  float p[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) p[k] = valid ? zyx[i * 3 + k] : 0.f;
  const int64_t row = valid ? i : 0;
  scatter_warp<3, F, false, true, S, true>(g, grad, p, valid, dout + row * ld, F, 1, 0u, l0, l1);
}

// Gradient of one hashed level of the (z, y, x) grid, restricted to the
// corners whose entry lies in half `half` of the level (entry >> shift ==
// half): two such passes keep each pass's reductions within 67 MB of a 2^23 x 4
// fp32 level, which L2 holds, where the whole level (134 MB) does not.  No run
// merging (hashed levels' samples rarely share cells).
template <int F, typename S>
__global__ void volume_scatter_half_kernel(GridDev g, const float* __restrict__ zyx, int64_t n,
                                           const S* __restrict__ dout, int64_t ld, float* __restrict__ grad, int l,
                                           int shift, uint32_t half) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x[3] = {zyx[i * 3], zyx[i * 3 + 1], zyx[i * 3 + 2]};
  LevelCorners<3> lc;
  level_corners<3>(g, l, x, lc);
  float d[F];
  load_grad_row<F, S>(dout + i * ld + l * F, d);
  float* base = grad + g.offset[l] * F;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    if ((lc.idx[c] >> shift) != half) continue;
    float v[F];
#pragma unroll
    for (int f = 0; f < F; ++f) v[f] = lc.w[c] * d[f];
    red_entry<F>(base + (int64_t)lc.idx[c] * F, v);
  }
}

// Gradient of a plane grid into the plane-shaped fp32 gradient: 4 corners a
// level; on levels where a warp's 32 points form at most 24 runs of equal
// cells, each run's sums are reduced once by its first lane.
template <int F, typename S>
__global__ void plane_scatter_kernel(Plane s, const float* __restrict__ zyx, int64_t n, int ca, int cb,
                                     const S* __restrict__ dout, int64_t ld, int col0, float* __restrict__ pgrad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const int lane = threadIdx.x & 31;
  const float a = valid ? zyx[i * 3 + ca] : 0.f, b = valid ? zyx[i * 3 + cb] : 0.f;
  const S* src = dout + (valid ? i : 0) * ld + col0;
#pragma unroll 1
  for (int l = 0; l < s.n_levels; ++l) {
    PlaneCorners pc;
    plane_corners(s, l, a, b, pc);
    float d[F];
    if (valid) {
      load_grad_row<F, S>(src + l * F, d);
    } else {
#pragma unroll
      for (int f = 0; f < F; ++f) d[f] = 0.f;
    }
    float* base = pgrad + s.off2[l] * F;
    const uint64_t key = valid ? pc.cell : ~uint64_t(0);
    const uint64_t prev = __shfl_up_sync(0xffffffffu, key, 1);
    const bool head = (lane == 0) || (prev != key);
    const uint32_t heads = __ballot_sync(0xffffffffu, head);
    if (__popc(heads) <= 24) {
      const uint32_t later = heads & ~((2u << lane) - 1u);
      const int end = later ? (__ffs(later) - 2) : 31;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float v[F];
#pragma unroll
        for (int f = 0; f < F; ++f) v[f] = run_sum(pc.w[q] * d[f], lane, end);
        if (head && valid) red_entry<F>(base + (int64_t)pc.idx[q] * F, v);
      }
    } else if (valid) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float v[F];
#pragma unroll
        for (int f = 0; f < F; ++f) v[f] = pc.w[q] * d[f];
        red_entry<F>(base + (int64_t)pc.idx[q] * F, v);
      }
    }
  }
}

// Adds the plane-shaped gradient to the 3D gradient table at the two time
// vertices (grid y = level).  Plane levels keyed by the hash: one thread per
// 3D entry e gathers plane entries e ^ c0 and e ^ c1 (an XOR is its own
// inverse, so every 3D entry has one writer).  Dense plane levels: one thread
// per non-zero plane entry; on dense 3D levels its two vertices are its own
// (different t slabs), on hashed ones they may collide and are reduced
// atomically.
template <int F>
__global__ void plane_spread_kernel(Plane s, const float* __restrict__ t, const float* __restrict__ pgrad,
                                    float* __restrict__ grad) {
  const int l = blockIdx.y;
  const TimeVertex tv = time_vertex(__ldg(t), s.res[l]);
  const float* src = pgrad + s.off2[l] * F;
  float* dst = grad + s.off3[l] * F;
  const bool hashed2 = (s.hashed2 >> l) & 1u, hashed3 = (s.hashed3 >> l) & 1u;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < s.n2[l];
       k += (int64_t)gridDim.x * blockDim.x) {
    if (hashed2) {
      int64_t j0, j1;   // the plane entries whose vertices are 3D entry k
      plane_sources(s, l, k, tv.c, &j0, &j1);
      float g0[F], g1[F];
      Feat<F, float>::load(src, j0, g0);
      Feat<F, float>::load(src, j1, g1);
      bool any = false;
#pragma unroll
      for (int f = 0; f < F; ++f) any |= (g0[f] != 0.f) | (g1[f] != 0.f);
      if (!any) continue;
#pragma unroll
      for (int f = 0; f < F; ++f) dst[k * F + f] += fmaf(tv.w0, g0[f], tv.w1 * g1[f]);
      continue;
    }
    float g[F];
    Feat<F, float>::load(src, k, g);
    bool any = false;
#pragma unroll
    for (int f = 0; f < F; ++f) any |= g[f] != 0.f;
    if (!any) continue;
    int64_t e0, e1;
    plane_sources(s, l, k, tv.c, &e0, &e1);
    float v0[F], v1[F];
#pragma unroll
    for (int f = 0; f < F; ++f) {
      v0[f] = tv.w0 * g[f];
      v1[f] = tv.w1 * g[f];
    }
    if (hashed3) {
      red_entry<F>(dst + e0 * F, v0);
      red_entry<F>(dst + e1 * F, v1);
    } else {
#pragma unroll
      for (int f = 0; f < F; ++f) {
        dst[e0 * F + f] += v0[f];
        dst[e1 * F + f] += v1[f];
      }
    }
  }
}

// The plane grids in the reference's input order (networks.py:438-446):
// (y, x, t), (x, z, t), (z, y, t); the (a, b) columns of zyx.
constexpr int kPlaneCols[3][2] = {{1, 2}, {2, 0}, {0, 1}};

dim3 plane_grid(const Plane& s) {
  int64_t widest = 0;
  for (int l = 0; l < s.n_levels; ++l) widest = std::max(widest, s.n2[l]);
  return dim3((unsigned)std::min<int64_t>(ceil_div(widest, 256), 4096), (unsigned)s.n_levels);
}

size_t plane_bytes(const Plane& s, int F) { return ((size_t)s.total2 * F * 4 + 255) & ~size_t(255); }

int check_grid(const NectbHashGrid* grid, GridDev* g, Plane* s) {
  if (!make_grid_dev(grid, g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  NECTB_REQUIRE(grid->n_dims == 3 && grid->feature_dtype == NECTB_F32,
                "QuadCubes grids are 3D with fp32 tables");
  NECTB_REQUIRE(grid->n_features == 2 || grid->n_features == 4, "n_features must be 2 or 4");
  NECTB_REQUIRE(make_plane(*g, s), "QuadCubes grids need the same resolution on every axis");
  return NECTB_OK;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

template <int F, typename P, typename O>
int encode_all(const GridDev& g, const Plane& s, const float* const* tables, const float* zyx, int64_t n,
               const float* t, int identity, O* out, int64_t ld, P* plane, cudaStream_t st) {
  const unsigned blocks = (unsigned)ceil_div(n, 256);
  const int LF = g.n_levels * F;
  volume_encode_kernel<F, O><<<blocks, 256, 0, st>>>(g, tables[0], zyx, t, n, identity, out, ld,
                                                     4 * LF + (identity ? 4 : 0));
  if (int rc = launch_status("volume_encode_kernel")) return rc;
  for (int k = 0; k < 3; ++k) {
    plane_build_kernel<F, P><<<plane_grid(s), 256, 0, st>>>(s, tables[k + 1], t, plane);
    if (int rc = launch_status("plane_build_kernel")) return rc;
    plane_encode_kernel<F, P, O><<<blocks, 256, 0, st>>>(s, plane, zyx, n, kPlaneCols[k][0], kPlaneCols[k][1], out,
                                                          ld, (k + 1) * LF);
    if (int rc = launch_status("plane_encode_kernel")) return rc;
  }
  return NECTB_OK;
}

constexpr int64_t kScatterGroupBytes = int64_t(64) << 20;

template <int F, typename S>
int backward_all(const GridDev& g, const Plane& s, const float* zyx, int64_t n, const float* t, const S* dout,
                 int64_t ld, float* const* grads, float* pgrad, cudaStream_t st) {
  const unsigned blocks = (unsigned)ceil_div(n, 256);
  const int LF = g.n_levels * F;
  // One pass per group of consecutive levels whose gradient slice is at most
  // kScatterGroupBytes (a hashed level of 2^23 entries is a group of its own),
  // so that a pass's reductions find their lines in L2 and each line is
  // written back about once; the passes re-read the points and their rows.
  for (int l0 = 0; l0 < g.n_levels;) {
    int l1 = l0 + 1;
    auto level_bytes = [&](int l) {
      const int64_t end = l + 1 < g.n_levels ? g.offset[l + 1] : g.total_entries;
      return (end - g.offset[l]) * F * 4;
    };
    int64_t bytes = level_bytes(l0);
    while (l1 < g.n_levels && bytes + level_bytes(l1) <= kScatterGroupBytes) bytes += level_bytes(l1++);
    if (l1 == l0 + 1 && ((g.hashed_bits >> l0) & 1u) && bytes > kScatterGroupBytes) {
      // a hashed level above the group size: one pass per half of its entries
      int log2T = 0;
      while ((1u << log2T) < g.hash_mask + 1u) ++log2T;
      for (uint32_t h = 0; h < 2; ++h) {
        volume_scatter_half_kernel<F, S><<<blocks, 256, 0, st>>>(g, zyx, n, dout, ld, grads[0], l0, log2T - 1, h);
        if (int rc = launch_status("volume_scatter_half_kernel")) return rc;
      }
    } else {
      volume_scatter_kernel<F, S><<<blocks, 256, 0, st>>>(g, zyx, n, dout, ld, grads[0], l0, l1);
      if (int rc = launch_status("volume_scatter_kernel")) return rc;
    }
    l0 = l1;
  }
  for (int k = 0; k < 3; ++k) {
    if (int rc = cuda_status(cudaMemsetAsync(pgrad, 0, (size_t)s.total2 * F * 4, st), "cudaMemsetAsync")) return rc;
    plane_scatter_kernel<F, S><<<blocks, 256, 0, st>>>(s, zyx, n, kPlaneCols[k][0], kPlaneCols[k][1], dout, ld,
                                                        (k + 1) * LF, pgrad);
    if (int rc = launch_status("plane_scatter_kernel")) return rc;
    plane_spread_kernel<F><<<plane_grid(s), 256, 0, st>>>(s, t, pgrad, grads[k + 1]);
    if (int rc = launch_status("plane_spread_kernel")) return rc;
  }
  return NECTB_OK;
}

}  // namespace
}  // namespace nectb

using namespace nectb;

extern "C" size_t nectb_quadcubes_workspace_bytes(const NectbHashGrid* grid) {
  GridDev g;
  Plane s;
  if (!grid || !make_grid_dev(grid, &g) || !make_plane(g, &s)) return 0;
  return plane_bytes(s, grid->n_features);
}

extern "C" int nectb_quadcubes_encode(const NectbHashGrid* grid, const float* const* tables, const float* zyx,
                                      int64_t n, const float* t, int identity, void* out, int64_t out_ld,
                                      int out_dtype, void* workspace, size_t workspace_bytes, void* stream) {
  clear_error();
  GridDev g;
  Plane s;
  if (int rc = check_grid(grid, &g, &s)) return rc;
  NECTB_REQUIRE(n >= 0, "negative size");
  if (n == 0) return NECTB_OK;
  NECTB_REQUIRE(tables && zyx && t && out && workspace, "null pointer");
  for (int k = 0; k < 4; ++k) NECTB_REQUIRE(tables[k] && aligned16(tables[k]), "tables must be 16-byte aligned");
  NECTB_REQUIRE(out_dtype == NECTB_F32 || out_dtype == NECTB_BF16, "out_dtype must be NECTB_F32 or NECTB_BF16");
  const int F = grid->n_features;
  const size_t esz = out_dtype == NECTB_F32 ? 4 : 2;
  NECTB_REQUIRE(out_ld >= 4 * (int64_t)g.n_levels * F + (identity ? 4 : 0), "out_ld narrower than a row");
  NECTB_REQUIRE(aligned16(out) && (out_ld * esz) % 16 == 0, "out and its rows must be 16-byte aligned");
  NECTB_REQUIRE(aligned16(workspace), "workspace must be 16-byte aligned");
  if (workspace_bytes < plane_bytes(s, F))
    return set_error(NECTB_ERR_WORKSPACE, "workspace %zu bytes < %zu", workspace_bytes, plane_bytes(s, F));
  cudaStream_t st = (cudaStream_t)stream;
  ProfScope ps(kProfModel, st);
  const int id = identity ? 1 : 0;
  if (out_dtype == NECTB_F32) {
    float* o = (float*)out;
    float* pl = (float*)workspace;
    return F == 2 ? encode_all<2>(g, s, tables, zyx, n, t, id, o, out_ld, pl, st)
                  : encode_all<4>(g, s, tables, zyx, n, t, id, o, out_ld, pl, st);
  }
  __nv_bfloat16* o = (__nv_bfloat16*)out;
  __half* pl = (__half*)workspace;
  return F == 2 ? encode_all<2>(g, s, tables, zyx, n, t, id, o, out_ld, pl, st)
                : encode_all<4>(g, s, tables, zyx, n, t, id, o, out_ld, pl, st);
}

extern "C" int nectb_quadcubes_encode_backward(const NectbHashGrid* grid, const float* zyx, int64_t n,
                                               const float* t, const void* dout, int64_t dout_ld, int dout_dtype,
                                               float* const* grads, void* workspace, size_t workspace_bytes,
                                               void* stream) {
  clear_error();
  GridDev g;
  Plane s;
  if (int rc = check_grid(grid, &g, &s)) return rc;
  NECTB_REQUIRE(n >= 0, "negative size");
  if (n == 0) return NECTB_OK;
  NECTB_REQUIRE(zyx && t && dout && grads && workspace, "null pointer");
  for (int k = 0; k < 4; ++k) NECTB_REQUIRE(grads[k] && aligned16(grads[k]), "grads must be 16-byte aligned");
  NECTB_REQUIRE(dout_dtype == NECTB_F32 || dout_dtype == NECTB_BF16, "dout_dtype must be NECTB_F32 or NECTB_BF16");
  const int F = grid->n_features;
  NECTB_REQUIRE(dout_ld >= 4 * (int64_t)g.n_levels * F, "dout_ld narrower than the four grids' columns");
  NECTB_REQUIRE(aligned16(dout) && (dout_ld * (dout_dtype == NECTB_F32 ? 4 : 2)) % 16 == 0,
                "dout and its rows must be 16-byte aligned");
  NECTB_REQUIRE(aligned16(workspace), "workspace must be 16-byte aligned");
  if (workspace_bytes < plane_bytes(s, F))
    return set_error(NECTB_ERR_WORKSPACE, "workspace %zu bytes < %zu", workspace_bytes, plane_bytes(s, F));
  cudaStream_t st = (cudaStream_t)stream;
  ProfScope ps(kProfModel, st);
  float* pg = (float*)workspace;
  if (dout_dtype == NECTB_F32) {
    const float* d = (const float*)dout;
    return F == 2 ? backward_all<2>(g, s, zyx, n, t, d, dout_ld, grads, pg, st)
                  : backward_all<4>(g, s, zyx, n, t, d, dout_ld, grads, pg, st);
  }
  const __nv_bfloat16* d = (const __nv_bfloat16*)dout;
  return F == 2 ? backward_all<2>(g, s, zyx, n, t, d, dout_ld, grads, pg, st)
                : backward_all<4>(g, s, zyx, n, t, d, dout_ld, grads, pg, st);
}
