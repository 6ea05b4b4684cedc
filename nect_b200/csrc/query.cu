// Query kernels: slice / volume points and detector re-projections of a
// trained model.
//
// nectb_query_points runs one persistent launch over the 128-point chunks of
// any number of work items (slices, volume slabs) of any number of requests:
// each block takes chunks from an atomic cursor, finds the chunk's item by
// binary search over the items' chunk offsets, generates the points from the
// item's origin and step vectors (no coordinate arrays in memory), evaluates
// the model and writes de-normalised values.  The mixed model runs its MLP on
// tcgen05 (the forward tile of the training kernel); the plain model the fp32
// SIMT MLP.  nectb_query_reproject reuses the fused training forward over all
// detector pixels of a view.
#include <algorithm>

#include "mixed_common.cuh"
#include "train_common.cuh"

namespace nectb {

int validate_geometry(const NectbGeometry* g);
int validate_mlp(const NectbMLP* m, const GridDev& g);
int64_t mlp_param_count(const NectbMLP* m);
int train_forward_only(const NectbGeometry& geo, const GridDev& grid, const NectbMLP& mlp, const void* table,
                       const float* W, const TrainArgs& a, Workspace ws, float* y_pred, float* loss, cudaStream_t s);
int launch_time_slice(const GridDev& grid, const __half* table, float t, __half* slice, cudaStream_t s);

namespace {

constexpr int kQThreads = 128;
constexpr uint32_t kQTile = 128 * 128;
constexpr uint32_t kQWTile = 64 * 128;

__device__ __forceinline__ int find_item(const NectbQueryItem* __restrict__ items, int n, int64_t chunk) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].chunk_begin <= chunk)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

struct QPoint {
  float p[4];
  bool valid;
  float* dst;
  float scale, offset;
};

__device__ __forceinline__ QPoint query_point(const NectbQueryItem& it, int64_t chunk, int t) {
  QPoint q;
  const int64_t k = (chunk - it.chunk_begin) * 128 + t;
  const int64_t n = (int64_t)it.nu * it.nv;
  q.valid = k < n;
  q.p[0] = q.p[1] = q.p[2] = 0.f;
  q.p[3] = it.t;
  q.dst = nullptr;
  q.scale = it.out_scale;
  q.offset = it.out_offset;
  if (q.valid) {
    const int i = (int)(k % it.nu), j = (int)(k / it.nu);
#pragma unroll
    for (int a = 0; a < 3; ++a) q.p[a] = clamp01f(it.origin[a] + (float)i * it.du[a] + (float)j * it.dv[a]);
    q.dst = it.out + (int64_t)j * it.out_stride + i;
  }
  return q;
}

__device__ __forceinline__ uint8_t* qalign1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// At most 128 registers so that three blocks share an SM under the 164 KB
// shared split (a background block beside two slice blocks, or three blocks of
// one query).
template <int D, int F, int L, int H, int ACT>
__global__ void __launch_bounds__(kQThreads, 4)
query_mixed_kernel(GridDev grid, const __half* __restrict__ table, const float* __restrict__ W,
                   const NectbQueryItem* __restrict__ items, int n_items, int64_t total_chunks,
                   unsigned int* __restrict__ counter, int out_act) {
  using S = InShape<L, F>;
  constexpr int KT = S::KT;
  constexpr int act = ACT;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = qalign1024(smem_raw);
  uint8_t* sW = base;                   // KT + H - 1 weight tiles
  uint8_t* sX = sW + (KT + H - 1) * kQWTile;
  uint8_t* sA = sX + KT * kQTile;       // every hidden layer's activations in turn
  float* sWout = reinterpret_cast<float*>(sA + kQTile);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sWout + 64);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  long long* s_chunk = reinterpret_cast<long long*>(tslot + 2);
  int* s_item = reinterpret_cast<int*>(s_chunk + 1);

  const int t = threadIdx.x, warp = t >> 5;
  // fp32 weights -> bf16 swizzled tiles (same layout as the training kernels)
  stage_mixed_weights<L, F, H>(W, sW, sWout);
  if (warp == 0) {
    tc::tmem_alloc(tslot, 128);
    tc::tmem_relinquish();
  }
  if (t == 0) tc::mbar_init(bar, 1);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tm = *tslot;
  const uint32_t my_lanes = tm + ((uint32_t)(32 * warp) << 16);
  const uint32_t sX_a = tc::smem_u32(sX), sA_a = tc::smem_u32(sA), sW_a = tc::smem_u32(sW);
  constexpr uint32_t idesc = tc::idesc_bf16(128, 64, false, false);
  uint32_t phase = 0;
  bool timed_out = false;
  while (true) {
    if (t == 0) {
      const long long c = (long long)atomicAdd(counter, 1u);
      *s_chunk = c;
      *s_item = c < total_chunks ? find_item(items, n_items, c) : 0;
    }
    __syncthreads();
    const long long chunk = *s_chunk;
    if (chunk >= total_chunks) break;
    const QPoint q = query_point(items[*s_item], chunk, t);
    encode_row<D, F, L>(grid, table, q.p, q.valid, sX, t);   // the encoder's row writer (fp16 gathers, bf16 row)
    // layer k writes TMEM columns 64 * (k & 1); its input is X for k = 0, else
    // the previous layer's activations in sA (written once the MMA that read
    // sA before has completed)
    float h[64];
#pragma unroll
    for (int k = 0; k < H; ++k) {
      if (k > 0) {
        uint32_t mlo, mhi;
        act_row(h, sA, t, act, mlo, mhi);
      }
      tc::fence_async_smem();
      tc::fence_before();
      __syncthreads();
      if (t == 0) {
        tc::fence_after();
        if (k == 0) {
#pragma unroll
          for (int c = 0; c < S::INP / 16; ++c)
            tc::mma(tm, tc::desc_k(sX_a + (c / 4) * kQTile, c % 4), tc::desc_k(sW_a + (c / 4) * kQWTile, c % 4),
                    idesc, c > 0);
        } else {
#pragma unroll
          for (int c = 0; c < 4; ++c)
            tc::mma(tm + 64 * (k & 1), tc::desc_k(sA_a, c), tc::desc_k(sW_a + (KT + k - 1) * kQWTile, c), idesc,
                    c > 0);
        }
        tc::commit(bar);
      }
      timed_out = !tc::mbar_wait(bar, phase);
      phase ^= 1;
      if (__syncthreads_or(timed_out)) {
        timed_out = true;
        break;
      }
      tc::fence_after();
#pragma unroll
      for (int c = 0; c < 4; ++c) tc::tmem_ld16(my_lanes + 64 * (k & 1) + 16 * c, h + 16 * c);
      tc::tmem_wait_ld();
    }
    if (timed_out) break;
    float z = 0.f;
#pragma unroll
    for (int j = 0; j < 64; ++j) z = fmaf(sWout[j], hidden_act(h[j], act), z);
    if (q.valid) *q.dst = fmaf(act_fwd(z, out_act), q.scale, q.offset);
    tc::fence_before();
    __syncthreads();
  }
  if (timed_out) {
    tc::mbar_wait(bar, phase);  // let the MMA in flight finish before TMEM is freed
    if (t == 0) atomicOr(counter + 1, 1u);
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(tm, 128);
  }
}

template <int D, int F, typename T, int L, int H>
__global__ void __launch_bounds__(kQThreads)
query_plain_kernel(GridDev grid, const T* __restrict__ table, const float* __restrict__ W,
                   const NectbQueryItem* __restrict__ items, int n_items, int64_t total_chunks,
                   unsigned int* __restrict__ counter, int act, int out_act) {
  constexpr int IN = L * F;
  constexpr int LD = kQThreads + 4;
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const SimtWeights sw = stage_weights<IN, H, false>(W, smem);
  float* xe = smem + simt_weight_floats<IN, H, false>() + threadIdx.x;
  float* hid = xe + IN * LD;  // two [64][LD] buffers, alternating between layers
  __shared__ long long s_chunk;
  __shared__ int s_item;
  const int t = threadIdx.x;
  __syncthreads();
  while (true) {
    if (t == 0) {
      const long long c = (long long)atomicAdd(counter, 1u);
      s_chunk = c;
      s_item = c < total_chunks ? find_item(items, n_items, c) : 0;
    }
    __syncthreads();
    const long long chunk = s_chunk;
    if (chunk >= total_chunks) break;
    const QPoint q = query_point(items[s_item], chunk, t);
    if (q.valid) {
      encode_point<D, F, T>(grid, table, q.p, xe, LD);
      float z;
      if (H == 1) {
        z = gemv_dot<IN, LD>(sw.WT[0], xe, sw.wout, act);
      } else {
        gemv_cols<IN, kWidth, LD>(sw.WT[0], xe, hid, act);
#pragma unroll
        for (int k = 1; k < H - 1; ++k)
          gemv_cols<kWidth, kWidth, LD>(sw.WT[k], hid + ((k - 1) & 1) * kWidth * LD, hid + (k & 1) * kWidth * LD,
                                        act);
        z = gemv_dot<kWidth, LD>(sw.WT[H - 1], hid + ((H - 2) & 1) * kWidth * LD, sw.wout, act);
      }
      *q.dst = fmaf(act_fwd(z, out_act), q.scale, q.offset);
    }
    __syncthreads();
  }
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <int D, int F, int L, int H, int ACT>
int launch_query_mixed(const GridDev& g, const void* table, const float* W, const NectbQueryItem* items, int n,
                       int64_t chunks, unsigned int* counter, int oact, int max_blocks, cudaStream_t s) {
  using S = InShape<L, F>;
  auto k = query_mixed_kernel<D, F, L, H, ACT>;
  const size_t smem = 1024 + (S::KT + H - 1) * kQWTile + (S::KT + 1) * kQTile + 64 * 4 + 64;
  set_smem(k, smem, true);
  int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(chunks, 3 * sm_count()));
  if (max_blocks > 0) blocks = std::min(blocks, max_blocks);
  GridDev gt = g;  // with a texture over the table for the gathers
  gt.tex = table_texture(table, (size_t)g.total_entries * F * sizeof(__half), F * (int)sizeof(__half));
  ProfScope ps(kProfModel, s);
  k<<<blocks, kQThreads, smem, s>>>(gt, (const __half*)table, W, items, n, chunks, counter, oact);
  return launch_status("query_mixed_kernel");
}

template <int D, int F, typename T, int L, int H>
int launch_query_plain(const GridDev& g, const void* table, const float* W, const NectbQueryItem* items, int n,
                       int64_t chunks, unsigned int* counter, int act, int oact, int max_blocks, cudaStream_t s) {
  constexpr int IN = L * F;
  auto k = query_plain_kernel<D, F, T, L, H>;
  const size_t smem =
      (size_t)(simt_weight_floats<IN, H, false>() + (IN + simt_hidden_buffers<H>() * kWidth) * (kQThreads + 4)) * 4;
  set_smem(k, smem, true);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kQThreads, smem);
  int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(chunks, (int64_t)sm_count() * std::max(per_sm, 1)));
  if (max_blocks > 0) blocks = std::min(blocks, max_blocks);
  ProfScope ps(kProfModel, s);
  k<<<blocks, kQThreads, smem, s>>>(g, (const T*)table, W, items, n, chunks, counter, act, oact);
  return launch_status("query_plain_kernel");
}

}  // namespace
}  // namespace nectb

using namespace nectb;

namespace {

// Items of one launch on grid g (a 3D or 4D table, or the 3D view of a 4D
// table's time slice).
int query_points_impl(const GridDev& g, bool f16_table, const NectbMLP* mlp, const void* grid_params,
                      const float* mlp_params, const NectbQueryItem* items, int32_t n_items, int64_t total_chunks,
                      unsigned int* counter, int32_t max_blocks, cudaStream_t s) {
  if (int rc = validate_mlp(mlp, g)) return rc;
  if (n_items == 0 || total_chunks == 0) return NECTB_OK;
  NECTB_REQUIRE(grid_params && mlp_params && items && counter && n_items > 0 && total_chunks > 0,
                "null pointer or empty query");
  NECTB_REQUIRE(total_chunks < (int64_t(1) << 31), "too many chunks in one launch");
  NECTB_REQUIRE(((uintptr_t)grid_params & 15u) == 0, "grid_params must be 16-byte aligned");
  if (int rc = cuda_status(cudaMemsetAsync(counter, 0, sizeof(unsigned int), s), "memset query counter")) return rc;
  const int D = g.n_dims, F = g.n_features, L = g.n_levels, H = mlp->n_hidden_layers;
  const int act = mlp->activation, oact = mlp->output_activation;
  const bool mixed = mlp->compute_dtype != NECTB_F32;
  if (mixed) {
    NECTB_REQUIRE(f16_table, "mixed queries need an fp16 table");
    NECTB_REQUIRE(H >= 2, "mixed queries need at least 2 hidden layers");
    const int rc = dispatch_shape(D, F, L, H, [&](auto d, auto f, auto l, auto h) {
      if (act == NECTB_ACT_RELU)
        return launch_query_mixed<d(), f(), l(), h(), NECTB_ACT_RELU>(g, grid_params, mlp_params, items, n_items,
                                                                       total_chunks, counter, oact, max_blocks, s);
      if constexpr (l() != 16) {
        if (act == NECTB_ACT_LEAKY_RELU)
          return launch_query_mixed<d(), f(), l(), h(), NECTB_ACT_LEAKY_RELU>(
              g, grid_params, mlp_params, items, n_items, total_chunks, counter, oact, max_blocks, s);
      }
      return set_error(NECTB_ERR_INVALID, "mixed queries: hidden activation %d is not instantiated for this shape",
                       act);
    });
    if (rc != kUnsupportedShape) return rc;
  } else {
    const int rc = dispatch_shape(D, F, L, H, [&](auto d, auto f, auto l, auto hl) {
      return f16_table ? launch_query_plain<d(), f(), __half, l(), hl()>(g, grid_params, mlp_params, items, n_items,
                                                                         total_chunks, counter, act, oact,
                                                                         max_blocks, s)
                       : launch_query_plain<d(), f(), float, l(), hl()>(g, grid_params, mlp_params, items, n_items,
                                                                        total_chunks, counter, act, oact,
                                                                        max_blocks, s);
    });
    if (rc != kUnsupportedShape) return rc;
  }
  return set_error(NECTB_ERR_INVALID, "queries: unsupported configuration (n_dims %d, n_features %d, n_levels %d, "
                   "hidden %d)", D, F, L, H);
}

// A 4D fp16 grid's slice layout, or false.
bool slice_grid(const NectbHashGrid* grid, GridDev* g3) {
  GridDev g;
  if (!grid || grid->n_dims != 4 || grid->feature_dtype != NECTB_F16 || !make_grid_dev(grid, &g)) return false;
  *g3 = make_time_slice(g, 0.f).g3;
  return true;
}

}  // namespace

extern "C" int nectb_query_points(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                                  const float* mlp_params, const NectbQueryItem* items, int32_t n_items,
                                  int64_t total_chunks, unsigned int* counter, int32_t max_blocks, void* stream) {
  clear_error();
  GridDev g;
  if (!make_grid_dev(grid, &g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  return query_points_impl(g, grid->feature_dtype == NECTB_F16, mlp, grid_params, mlp_params, items, n_items,
                           total_chunks, counter, max_blocks, (cudaStream_t)stream);
}

extern "C" size_t nectb_time_slice_bytes(const NectbHashGrid* grid) {
  GridDev g3;
  if (!slice_grid(grid, &g3)) return 0;
  return (size_t)g3.total_entries * g3.n_features * 2;
}

extern "C" int nectb_time_slice(const NectbHashGrid* grid, const void* grid_params, float t, void* slice,
                                size_t slice_bytes, void* stream) {
  clear_error();
  GridDev g, g3;
  if (!slice_grid(grid, &g3) || !make_grid_dev(grid, &g))
    return set_error(NECTB_ERR_INVALID, "time slice: needs a valid 4D grid with an fp16 table");
  NECTB_REQUIRE(grid_params && slice, "null pointer");
  NECTB_REQUIRE(((uintptr_t)grid_params & 15u) == 0 && ((uintptr_t)slice & 15u) == 0,
                "grid_params and slice must be 16-byte aligned");
  NECTB_REQUIRE(t >= 0.f && t <= 1.f, "t must lie in [0, 1]");
  const size_t need = (size_t)g3.total_entries * g3.n_features * 2;
  if (slice_bytes < need) return set_error(NECTB_ERR_WORKSPACE, "slice of %zu bytes < required %zu", slice_bytes, need);
  return launch_time_slice(g, (const __half*)grid_params, t, (__half*)slice, (cudaStream_t)stream);
}

extern "C" int nectb_query_points_slice(const NectbHashGrid* grid, const NectbMLP* mlp, const void* slice,
                                        const float* mlp_params, const NectbQueryItem* items, int32_t n_items,
                                        int64_t total_chunks, unsigned int* counter, int32_t max_blocks,
                                        void* stream) {
  clear_error();
  GridDev g3;
  if (!slice_grid(grid, &g3))
    return set_error(NECTB_ERR_INVALID, "slice queries: needs a valid 4D grid with an fp16 table");
  return query_points_impl(g3, true, mlp, slice, mlp_params, items, n_items, total_chunks, counter, max_blocks,
                           (cudaStream_t)stream);
}

namespace {

// Pixels [begin, begin + count) of a re-projection at (angle, t), written to
// out[begin ...].  stage: use the workspace past the base size (a 4D mixed
// model's time slice).
int reproject_range(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                    const void* grid_params, const float* mlp_params, float angle_rad, float t,
                    int32_t num_points_per_ray, float max_ray_distance_per_point, float max_distance_traveled,
                    float* out, int32_t begin, int32_t count, void* workspace, size_t workspace_size,
                    int32_t max_blocks, int32_t warpgroups, bool stage, cudaStream_t s) {
  clear_error();
  if (int rc = validate_geometry(geometry)) return rc;
  GridDev g;
  if (!make_grid_dev(grid, &g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  if (int rc = validate_mlp(mlp, g)) return rc;
  NECTB_REQUIRE(grid_params && mlp_params && out, "null pointer");
  NECTB_REQUIRE(((uintptr_t)grid_params & 15u) == 0, "grid_params must be 16-byte aligned");
  NECTB_REQUIRE(num_points_per_ray >= 1 && max_distance_traveled > 0.f, "bad sampling parameters");
  const int P = geometry->nDetector[0] * geometry->nDetector[1];
  NECTB_REQUIRE(begin >= 0 && count >= 1 && (int64_t)begin + count <= P, "pixel range outside the detector");
  NECTB_REQUIRE(warpgroups >= 0 && warpgroups <= kFwdMaxWarpgroups, "warpgroups_per_sm must be 0..%d",
                kFwdMaxWarpgroups);
  if (!workspace || workspace_size < workspace_bytes(count, count))
    return set_error(NECTB_ERR_WORKSPACE, "workspace of %zu bytes < required %zu", workspace_size,
                     workspace_bytes(count, count));
  TrainArgs a;
  a.perm = nullptr;  // the pixels begin, begin + 1, ... in pixel order
  a.perm_len = count;
  a.start = begin;
  a.num_rays = count;
  a.n_pixels = count;
  a.S = num_points_per_ray;
  a.angle = angle_rad;
  a.t = t;
  a.maxd = max_ray_distance_per_point;
  a.uniform = 1;
  a.max_dist = max_distance_traveled;
  a.jitter = nullptr;
  a.det_off = nullptr;
  a.projection = nullptr;
  a.loss_type = 2;
  a.loss_scale = 0.f;
  a.max_blocks = max_blocks;
  a.fwd_warpgroups = max_blocks > 0 ? 0 : warpgroups;
  Workspace ws = carve_workspace(workspace, count, count, stage ? workspace_size : 0);
  float* y = out + begin;
  float* loss = reinterpret_cast<float*>(ws.counters + 8);
  if (int rc = cuda_status(cudaMemsetAsync(ws.counters, 0, 64, s), "memset counters")) return rc;
  if (int rc = cuda_status(cudaMemsetAsync(ws.slot, 0xFF, (size_t)count * 4, s), "memset slots")) return rc;
  {
    ProfScope ps(kProfRayPrep, s);
    ray_prep_kernel<<<(unsigned)ceil_div(count, 8), 256, 0, s>>>(*geometry, a, ws.rays, ws.slot, ws.counters, y,
                                                                  loss);
  }
  if (int rc = launch_status("ray_prep_kernel")) return rc;
  return train_forward_only(*geometry, g, *mlp, grid_params, mlp_params, a, ws, y, loss, s);
}

}  // namespace

extern "C" int nectb_query_reproject(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                                     const void* grid_params, const float* mlp_params, float angle_rad, float t,
                                     int32_t num_points_per_ray, float max_ray_distance_per_point,
                                     float max_distance_traveled, float* out, void* workspace,
                                     size_t workspace_size, int32_t max_blocks, void* stream) {
  const int P = geometry ? geometry->nDetector[0] * geometry->nDetector[1] : 0;
  return reproject_range(geometry, grid, mlp, grid_params, mlp_params, angle_rad, t, num_points_per_ray,
                         max_ray_distance_per_point, max_distance_traveled, out, 0, P, workspace, workspace_size,
                         max_blocks, 0, false, (cudaStream_t)stream);
}

extern "C" int nectb_query_reproject_range(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                           const NectbMLP* mlp, const void* grid_params, const float* mlp_params,
                                           float angle_rad, float t, int32_t num_points_per_ray,
                                           float max_ray_distance_per_point, float max_distance_traveled,
                                           float* out, int32_t pixel_begin, int32_t pixel_count, void* workspace,
                                           size_t workspace_size, int32_t max_blocks, int32_t warpgroups_per_sm,
                                           void* stream) {
  return reproject_range(geometry, grid, mlp, grid_params, mlp_params, angle_rad, t, num_points_per_ray,
                         max_ray_distance_per_point, max_distance_traveled, out, pixel_begin, pixel_count, workspace,
                         workspace_size, max_blocks, warpgroups_per_sm, true, (cudaStream_t)stream);
}

extern "C" size_t nectb_query_reproject_slice_bytes(const NectbHashGrid* grid, const NectbMLP* mlp,
                                                    int32_t pixel_count) {
  GridDev g;
  if (!grid || !mlp || pixel_count < 1 || !make_grid_dev(grid, &g)) return 0;
  if (g.n_dims != 4 || mlp->compute_dtype == NECTB_F32 || grid->feature_dtype != NECTB_F16) return 0;
  return slice_half_bytes(g) + 512;
}
