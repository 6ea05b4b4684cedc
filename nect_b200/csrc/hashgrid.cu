// Hash-grid layout, standalone encoding and model forward (queries/export).
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "hashgrid.cuh"
#include "mlp_simt.cuh"

namespace nectb {

bool make_grid_dev(const NectbHashGrid* g, GridDev* out) {
  if (!g || (g->n_dims != 3 && g->n_dims != 4) || g->n_levels < 1 || g->n_levels > NECTB_MAX_LEVELS ||
      g->n_features < 1 || g->log2_hashmap_size < 4 || g->log2_hashmap_size > 30 || !(g->base_resolution >= 1.0) ||
      !(g->per_level_scale >= 1.0))
    return false;
  const int64_t T = int64_t(1) << g->log2_hashmap_size;
  out->n_dims = g->n_dims;
  out->n_levels = g->n_levels;
  out->n_features = g->n_features;
  out->hash_mask = (uint32_t)(T - 1);
  out->hashed_bits = 0;
  int64_t off = 0;
  for (int l = 0; l < g->n_levels; ++l) {
    const int r = (int)std::floor(g->base_resolution * std::pow(g->per_level_scale, (double)l));
    const double bt = g->base_resolution_t > 0 ? g->base_resolution_t : g->base_resolution;
    const int rt = (int)std::floor(bt * std::pow(g->per_level_scale, (double)l));
    int res[4] = {r, r, r, g->n_dims == 4 ? rt : 0};
    if (r < 1 || (g->n_dims == 4 && rt < 1)) return false;
    double verts = 1;
    uint32_t stride = 1;
    for (int k = 0; k < 4; ++k) {
      out->res[l][k] = res[k];
      if (k < g->n_dims) {
        out->stride[l][k] = stride;
        verts *= (double)(res[k] + 1);
        stride = (uint32_t)std::min<double>(verts, 4294967295.0);
      } else {
        out->stride[l][k] = 0;
      }
    }
    int64_t entries;
    if (verts <= (double)T) {
      entries = ((int64_t)verts + 7) / 8 * 8;
    } else {
      entries = T;
      out->hashed_bits |= 1u << l;
    }
    out->offset[l] = off;
    off += entries;
  }
  out->total_entries = off;
  return true;
}

namespace {

template <int D, int F, typename T>
__global__ void encode_kernel(GridDev g, const T* __restrict__ table, const float* __restrict__ x, int64_t n,
                              float* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float p[D];
#pragma unroll
  for (int k = 0; k < D; ++k) p[k] = x[i * D + k];
  encode_point<D, F, T>(g, table, p, out + i * (int64_t)g.n_levels * F);
}

// One thread per point: encode into a shared-memory column, then the SIMT MLP.
constexpr int kModelThreads = 128;

template <int D, int F, typename T, int IN, int H>
__global__ void __launch_bounds__(kModelThreads) model_forward_kernel(GridDev g, const T* __restrict__ table,
                                                                      const float* __restrict__ W,
                                                                      const float* __restrict__ x, int64_t n,
                                                                      float t, const float* __restrict__ t_dev,
                                                                      int act, int out_act,
                                                                      float* __restrict__ sigma) {
  constexpr int LD = kModelThreads + 4;
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const SimtWeights sw = stage_weights<IN, H, false>(W, smem);
  float* xe = smem + simt_weight_floats<IN, H, false>() + threadIdx.x;
  float* hid = xe + IN * LD;  // two [64][LD] buffers, alternating between layers
  if (D == 4 && t_dev) t = *t_dev;   // the broadcast timestep, read on the device
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float p[4];
#pragma unroll
    for (int k = 0; k < 3; ++k) p[k] = x[i * 3 + k];
    if (D == 4) p[3] = t;
    encode_point<D, F, T>(g, table, p, xe, LD);
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
    sigma[i] = act_fwd(z, out_act);
  }
}

// One thread per point: the point's encoding gradient dout[l * F + f] added
// to its corners' entries, weighted (fp32 vector atomics).  A warp's 32
// consecutive points merge their contributions on levels where they fall in
// runs of equal cells (consecutive samples of a ray do on the coarse levels),
// so such a run reduces each corner once.
template <int D, int F>
__global__ void encode_backward_kernel(GridDev g, const float* __restrict__ x, int64_t n,
                                       const float* __restrict__ dout, float* __restrict__ grad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool valid = i < n;   // every lane takes part in the warp's shuffles
  float p[D];
#pragma unroll
  for (int k = 0; k < D; ++k) p[k] = valid ? x[i * D + k] : 0.f;
  const int64_t row = valid ? i : 0;
  scatter_warp<D, F, false, true>(g, grad, p, valid, dout + row * (int64_t)g.n_levels * F, F, 1, 0u, 0,
                                  g.n_levels);
}

template <int D, int F, typename T>
int launch_encode(const GridDev& g, const void* params, const float* x, int64_t n, float* out, cudaStream_t s) {
  encode_kernel<D, F, T><<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(g, (const T*)params, x, n, out);
  return launch_status("encode_kernel");
}

template <int D, int F, typename T, int L, int H>
int launch_model(const GridDev& g, const void* params, const float* W, const float* x, int64_t n, float t,
                 const float* t_dev, int act, int out_act, float* sigma, cudaStream_t s) {
  constexpr int IN = L * F;
  auto k = model_forward_kernel<D, F, T, IN, H>;
  const size_t smem = (size_t)(simt_weight_floats<IN, H, false>() +
                               (IN + simt_hidden_buffers<H>() * kWidth) * (kModelThreads + 4)) * sizeof(float);
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kModelThreads, smem);
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, kModelThreads), (int64_t)sms * std::max(per_sm, 1)));
  ProfScope ps(kProfModel, s);
  k<<<blocks, kModelThreads, smem, s>>>(g, (const T*)params, W, x, n, t, t_dev, act, out_act, sigma);
  return launch_status("model_forward_kernel");
}

}  // namespace

int dispatch_encode(const GridDev& g, int dtype, const void* params, const float* x, int64_t n, float* out,
                    cudaStream_t s) {
  const bool h = dtype == NECTB_F16;
  if (g.n_dims == 3 && g.n_features == 2) return h ? launch_encode<3, 2, __half>(g, params, x, n, out, s)
                                                   : launch_encode<3, 2, float>(g, params, x, n, out, s);
  if (g.n_dims == 3 && g.n_features == 4) return h ? launch_encode<3, 4, __half>(g, params, x, n, out, s)
                                                   : launch_encode<3, 4, float>(g, params, x, n, out, s);
  if (g.n_dims == 4 && g.n_features == 2) return h ? launch_encode<4, 2, __half>(g, params, x, n, out, s)
                                                   : launch_encode<4, 2, float>(g, params, x, n, out, s);
  if (g.n_dims == 4 && g.n_features == 4) return h ? launch_encode<4, 4, __half>(g, params, x, n, out, s)
                                                   : launch_encode<4, 4, float>(g, params, x, n, out, s);
  return set_error(NECTB_ERR_INVALID, "unsupported grid (n_dims %d, n_features %d)", g.n_dims, g.n_features);
}

// Instantiated for the shapes of dispatch_shape, fp32 or fp16 tables.
int dispatch_model(const GridDev& g, int dtype, int H, const void* p, const float* W, const float* x, int64_t n,
                   float t, const float* t_dev, int act, int oact, float* sigma, cudaStream_t s) {
  const bool h = dtype == NECTB_F16;
  const int D = g.n_dims, F = g.n_features, L = g.n_levels;
  const int rc = dispatch_shape(D, F, L, H, [&](auto d, auto f, auto l, auto hl) {
    return h ? launch_model<d(), f(), __half, l(), hl()>(g, p, W, x, n, t, t_dev, act, oact, sigma, s)
             : launch_model<d(), f(), float, l(), hl()>(g, p, W, x, n, t, t_dev, act, oact, sigma, s);
  });
  if (rc != kUnsupportedShape) return rc;
  return set_error(NECTB_ERR_INVALID, "model forward: unsupported configuration (n_dims %d, n_features %d, "
                   "n_levels %d, hidden %d, %s table)", D, F, L, H, h ? "fp16" : "fp32");
}

int64_t mlp_param_count(const NectbMLP* m) {
  return (int64_t)m->width * m->n_input + (int64_t)(m->n_hidden_layers - 1) * m->width * m->width + m->width;
}

int validate_mlp(const NectbMLP* m, const GridDev& g) {
  NECTB_REQUIRE(m != nullptr, "mlp is null");
  NECTB_REQUIRE(m->width == kWidth, "only width 64 is supported (got %d)", m->width);
  NECTB_REQUIRE(m->n_hidden_layers >= 1 && m->n_hidden_layers <= kMaxHidden, "n_hidden_layers must be 1..%d",
                kMaxHidden);
  NECTB_REQUIRE(m->n_input == g.n_levels * g.n_features, "n_input %d != n_levels*n_features %d", m->n_input,
                g.n_levels * g.n_features);
  NECTB_REQUIRE(m->activation == NECTB_ACT_RELU || m->activation == NECTB_ACT_LEAKY_RELU ||
                    m->activation == NECTB_ACT_NONE,
                "hidden activation must be none, relu or leaky relu");
  return NECTB_OK;
}

}  // namespace nectb

using namespace nectb;

extern "C" int64_t nectb_hashgrid_layout(const NectbHashGrid* grid, int32_t* resolution, int32_t* resolution_t,
                                         int64_t* offset, int64_t* entries, int32_t* hashed) {
  GridDev g;
  if (!make_grid_dev(grid, &g)) return -1;
  for (int l = 0; l < g.n_levels; ++l) {
    if (resolution) resolution[l] = g.res[l][0];
    if (resolution_t) resolution_t[l] = g.n_dims == 4 ? g.res[l][3] : 0;
    if (offset) offset[l] = g.offset[l];
    if (entries) entries[l] = (l + 1 < g.n_levels ? g.offset[l + 1] : g.total_entries) - g.offset[l];
    if (hashed) hashed[l] = (g.hashed_bits >> l) & 1;
  }
  return g.total_entries;
}

extern "C" int64_t nectb_mlp_param_count(const NectbMLP* mlp) { return mlp ? mlp_param_count(mlp) : -1; }

extern "C" int nectb_hashgrid_encode(const NectbHashGrid* grid, const void* params, const float* x, int64_t n,
                                     float* out, void* stream) {
  clear_error();
  GridDev g;
  if (!make_grid_dev(grid, &g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  if (n == 0) return NECTB_OK;
  NECTB_REQUIRE(params && x && out && n > 0, "null pointer or negative size");
  return dispatch_encode(g, grid->feature_dtype, params, x, n, out, (cudaStream_t)stream);
}

extern "C" int nectb_hashgrid_encode_backward(const NectbHashGrid* grid, const float* x, int64_t n,
                                              const float* dout, float* grad, void* stream) {
  clear_error();
  GridDev g;
  if (!make_grid_dev(grid, &g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  if (n == 0) return NECTB_OK;
  NECTB_REQUIRE(x && dout && grad && n > 0, "null pointer or negative size");
  NECTB_REQUIRE(((uintptr_t)grad & 15u) == 0, "grad must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned blocks = (unsigned)ceil_div(n, 256);
  ProfScope ps(kProfModel, s);
  if (g.n_dims == 3 && g.n_features == 2)
    encode_backward_kernel<3, 2><<<blocks, 256, 0, s>>>(g, x, n, dout, grad);
  else if (g.n_dims == 3 && g.n_features == 4)
    encode_backward_kernel<3, 4><<<blocks, 256, 0, s>>>(g, x, n, dout, grad);
  else if (g.n_dims == 4 && g.n_features == 2)
    encode_backward_kernel<4, 2><<<blocks, 256, 0, s>>>(g, x, n, dout, grad);
  else if (g.n_dims == 4 && g.n_features == 4)
    encode_backward_kernel<4, 4><<<blocks, 256, 0, s>>>(g, x, n, dout, grad);
  else
    return set_error(NECTB_ERR_INVALID, "unsupported grid (n_dims %d, n_features %d)", g.n_dims, g.n_features);
  return launch_status("encode_backward_kernel");
}

namespace {
int model_forward_entry(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                        const float* mlp_params, const float* x, int64_t n, float t, const float* t_dev,
                        float* sigma, void* stream) {
  clear_error();
  GridDev g;
  if (!make_grid_dev(grid, &g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  if (int rc = validate_mlp(mlp, g)) return rc;
  if (n == 0) return NECTB_OK;
  NECTB_REQUIRE(grid_params && mlp_params && x && sigma && n > 0, "null pointer or negative size");
  return dispatch_model(g, grid->feature_dtype, mlp->n_hidden_layers, grid_params, mlp_params, x, n, t, t_dev,
                        mlp->activation, mlp->output_activation, sigma, (cudaStream_t)stream);
}
}  // namespace

extern "C" int nectb_model_forward(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                                   const float* mlp_params, const float* x, int64_t n, float t, float* sigma,
                                   void* stream) {
  return model_forward_entry(grid, mlp, grid_params, mlp_params, x, n, t, nullptr, sigma, stream);
}

extern "C" int nectb_model_forward_t(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                                     const float* mlp_params, const float* x, int64_t n, const float* t,
                                     float* sigma, void* stream) {
  if (!t) return set_error(NECTB_ERR_INVALID, "null timestep pointer");
  return model_forward_entry(grid, mlp, grid_params, mlp_params, x, n, 0.f, t, sigma, stream);
}

namespace nectb {
namespace {
template <int D>
__global__ void corners_kernel(GridDev g, const float* __restrict__ x, int64_t n, int32_t* __restrict__ idx,
                               float* __restrict__ w) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float p[D];
#pragma unroll
  for (int k = 0; k < D; ++k) p[k] = x[i * D + k];
  for (int l = 0; l < g.n_levels; ++l) {
    LevelCorners<D> lc;
    level_corners<D>(g, l, p, lc);
    const int64_t o = (i * g.n_levels + l) << D;
#pragma unroll
    for (int c = 0; c < (1 << D); ++c) {
      idx[o + c] = (int32_t)lc.idx[c];
      w[o + c] = lc.w[c];
    }
  }
}
}  // namespace
}  // namespace nectb

extern "C" int nectb_hashgrid_corners(const NectbHashGrid* grid, const float* x, int64_t n, int32_t* idx, float* w,
                                      void* stream) {
  clear_error();
  GridDev g;
  if (!make_grid_dev(grid, &g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  if (n == 0) return NECTB_OK;
  NECTB_REQUIRE(x && idx && w && n > 0, "null pointer or negative size");
  const unsigned blocks = (unsigned)ceil_div(n, 128);
  if (g.n_dims == 3)
    corners_kernel<3><<<blocks, 128, 0, (cudaStream_t)stream>>>(g, x, n, idx, w);
  else
    corners_kernel<4><<<blocks, 128, 0, (cudaStream_t)stream>>>(g, x, n, idx, w);
  return launch_status("corners_kernel");
}
