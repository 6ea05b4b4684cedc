// C-ABI entry points of the fused training step and the Adam update.
#include <algorithm>

#include "mlp_simt.cuh"
#include "train_common.cuh"

namespace nectb {

int validate_geometry(const NectbGeometry* g);
int validate_mlp(const NectbMLP* m, const GridDev& g);
int64_t mlp_param_count(const NectbMLP* m);
int train_plain(const NectbGeometry& geo, const GridDev& grid, const NectbMLP& mlp, const float* table,
                const float* W, int nW, const TrainArgs& a, Workspace ws, float* table_grad, float* W_grad,
                float* y_pred, float* loss, cudaStream_t s);
int train_mixed(const NectbGeometry& geo, const GridDev& grid, const NectbMLP& mlp, const void* table,
                const float* W, int nW, const TrainArgs& a, Workspace ws, float* table_grad, float* W_grad,
                float* y_pred, float* loss, cudaStream_t s);

int model_backward(const GridDev& g, const NectbMLP& mlp, int dtype, const void* table, const float* W,
                   const float* x, int64_t n, float tval, const float* t_dev, const float* dsigma, float* table_grad,
                   float* W_grad, cudaStream_t s);

namespace {

// torch.optim.Adam (no amsgrad, not maximize), in torch's order of
// operations: g += wd * p; m = lerp(m, g, 1 - b1);
// v = v * b2 + (1 - b2) * g * g; p += -(lr / bc1) * m / (sqrt(v) / sqrt(bc2) + eps).
// The host computes 1 - b1, 1 - b2, lr / bc1 and sqrt(bc2) in double, as torch
// does before casting its scalars to fp32.
struct AdamScalars {
  float w1, b2, w2, eps, wd, neg_step, bc2_sqrt;
};

// Every operation is pinned (explicit round-to-nearest intrinsics, no
// contraction left to the compiler), so both paths below give the same bits.
__device__ __forceinline__ float adam_element(const AdamScalars& c, float& param, float grad, float& m, float& v) {
  if (c.wd != 0.f) grad = __fmaf_rn(c.wd, param, grad);
  const float mi = __fmaf_rn(c.w1, __fsub_rn(grad, m), m);
  const float vi = __fmaf_rn(__fmul_rn(c.w2, grad), grad, __fmul_rn(v, c.b2));
  m = mi;
  v = vi;
  const float denom = __fadd_rn(__fdiv_rn(__fsqrt_rn(vi), c.bc2_sqrt), c.eps);
  param = __fmaf_rn(c.neg_step, __fdiv_rn(mi, denom), param);
  return param;
}

// Four elements per thread and iteration (16-byte loads and stores; p_half
// 8-byte aligned), then the n % 4 tail one element per thread.  HBM-bound:
// 28 bytes per element (32 with zero_grad, 30 with the fp16 copy).
__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, AdamScalars c, __half* __restrict__ p_half,
                            int zero_grad, int vec) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t n4 = vec ? n / 4 : 0;
  for (int64_t i = tid; i < n4; i += stride) {
    const float4 gq = reinterpret_cast<const float4*>(g)[i];
    float4 pq = reinterpret_cast<const float4*>(p)[i];
    float4 mq = reinterpret_cast<const float4*>(m)[i];
    float4 vq = reinterpret_cast<const float4*>(v)[i];
    adam_element(c, pq.x, gq.x, mq.x, vq.x);
    adam_element(c, pq.y, gq.y, mq.y, vq.y);
    adam_element(c, pq.z, gq.z, mq.z, vq.z);
    adam_element(c, pq.w, gq.w, mq.w, vq.w);
    reinterpret_cast<float4*>(m)[i] = mq;
    reinterpret_cast<float4*>(v)[i] = vq;
    reinterpret_cast<float4*>(p)[i] = pq;
    if (p_half) {
      const __half2 lo = __floats2half2_rn(pq.x, pq.y), hi = __floats2half2_rn(pq.z, pq.w);
      uint2 raw;
      raw.x = *reinterpret_cast<const unsigned int*>(&lo);
      raw.y = *reinterpret_cast<const unsigned int*>(&hi);
      reinterpret_cast<uint2*>(p_half)[i] = raw;
    }
    if (zero_grad) reinterpret_cast<float4*>(g)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int64_t i = n4 * 4 + tid; i < n; i += stride) {
    float param = p[i], mi = m[i], vi = v[i];
    adam_element(c, param, g[i], mi, vi);
    m[i] = mi;
    v[i] = vi;
    p[i] = param;
    if (p_half) p_half[i] = __float2half_rn(param);
    if (zero_grad) g[i] = 0.f;
  }
}

}  // namespace

// Forward kernels only (y_pred and loss; no gradients) after ray_prep_kernel
// has filled the workspace: used by re-projection queries.
int train_forward_only(const NectbGeometry& geo, const GridDev& grid, const NectbMLP& mlp, const void* table,
                       const float* W, const TrainArgs& a, Workspace ws, float* y_pred, float* loss,
                       cudaStream_t s) {
  const int nW = (int)mlp_param_count(&mlp);
  if (mlp.compute_dtype == NECTB_F32)
    return train_plain(geo, grid, mlp, (const float*)table, W, nW, a, ws, nullptr, nullptr, y_pred, loss, s);
  return train_mixed(geo, grid, mlp, table, W, nW, a, ws, nullptr, nullptr, y_pred, loss, s);
}

}  // namespace nectb

using namespace nectb;

extern "C" size_t nectb_train_workspace_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                              const NectbMLP* mlp, int32_t num_rays) {
  (void)grid;
  (void)mlp;
  const int P = geometry ? geometry->nDetector[0] * geometry->nDetector[1] : 0;
  return workspace_bytes(std::max(num_rays, 1), std::max(P, 0));
}

namespace nectb {
namespace {

// Warp per prepared ray: its count and scale, and (points non-null) the
// positions sample_point regenerates for samples 0..S-1, zeros past the count.
__global__ void train_rays_kernel(const RayRec* __restrict__ recs, int R, int S, int32_t* __restrict__ counts,
                                  float* __restrict__ scale, float* __restrict__ points) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= R) return;
  const RayRec rec = recs[r];
  if (lane == 0) {
    if (counts) counts[r] = rec.count;
    if (scale) scale[r] = rec.scale;
  }
  if (!points) return;
  float* out = points + (int64_t)r * S * 3;
  for (int i = lane; i < S; i += 32) {
    float p[3] = {0.f, 0.f, 0.f};
    if (i < rec.count) sample_point(rec, i, p);
    out[3 * i + 0] = p[0];
    out[3 * i + 1] = p[1];
    out[3 * i + 2] = p[2];
  }
}

// dL/dsigma of every sample of ray v is dL/dy_pred[r] * scale[v] / sub (y_pred
// is the scaled sum of the ray's sigmas, base_trainer.py:552-554; a
// continuous-scan step averages it over the sub angles of pixel r = v mod
// n_batch, continous_scanning_trainer.py:126-137).
__global__ void set_ray_grad_kernel(RayRec* __restrict__ recs, const float* __restrict__ dloss_dy, int R, int n_batch,
                                    int sub) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < R) recs[v].gsig = dloss_dy[v % n_batch] * recs[v].scale / (float)sub;
}

// Continuous scan, after the forward kernels wrote each virtual ray's
// integral: y_pred[r] = sum_j part[j * n + r] / sub in the reference's
// order (continous_scanning_trainer.py:126-137), the loss (mean over the n
// pixels) and, with grads, dL/dsigma of every virtual ray.
__global__ void scan_finalize_kernel(RayRec* __restrict__ recs, const float* __restrict__ part, int n, int sub,
                                     float* __restrict__ y_pred, float* __restrict__ loss, int loss_type,
                                     float loss_scale, int grads) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  float term = 0.f;
  if (r < n) {
    float y = 0.f;
    for (int j = 0; j < sub; ++j) y += part[(int64_t)j * n + r] / (float)sub;
    y_pred[r] = y;
    const float meas = recs[r].y;
    term = loss_term(y, meas, loss_type) / (float)n;
    if (grads) {
      const float g = loss_grad(y, meas, loss_type, n, 1.f) * loss_scale;
      for (int j = 0; j < sub; ++j) {
        RayRec& rec = recs[(int64_t)j * n + r];
        rec.gsig = g * rec.scale / (float)sub;
      }
    }
  }
  if (loss) {
    term = warp_sum(term);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, term);
  }
}

// Bytes of a continuous-scan workspace: the prepared virtual rays and pixel
// slots, then the per-virtual-ray integrals; staging follows.
size_t scan_workspace_bytes(int R, int P, int sub) {
  return align256(workspace_bytes(R * sub, P * sub)) + align256((size_t)R * sub * 4);
}

// The whole step (phase forward | backward, built-in loss), its forward half
// (y_pred only; the workspace keeps the prepared rays) or its backward half
// (dL/dy_pred given by the caller, the workspace of the matching forward).
// sub > 1: a continuous-scan step over sub_angles (host array of sub angles);
// the batch's jitter and detector offsets hold sub * num_rays entries,
// sub-angle-major.
int train_entry(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                const float* dloss_dy, float* grid_grad, float* mlp_grad, float* y_pred, float* loss,
                void* workspace, size_t workspace_size, void* stream, int phase, const float* sub_angles = nullptr,
                int sub = 1, bool texture = true) {
  clear_error();
  if (int rc = validate_geometry(geometry)) return rc;
  GridDev g;
  if (!make_grid_dev(grid, &g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  if (int rc = validate_mlp(mlp, g)) return rc;
  NECTB_REQUIRE(batch != nullptr, "batch is null");
  NECTB_REQUIRE(batch->num_rays >= 0 && batch->num_points_per_ray >= 1, "bad batch sizes");
  NECTB_REQUIRE(batch->loss_type == 1 || batch->loss_type == 2, "loss_type must be 1 (L1) or 2 (L2)");
  NECTB_REQUIRE(batch->max_distance_traveled > 0.f, "max_distance_traveled must be positive");
  NECTB_REQUIRE(grid_params && mlp_params, "null parameters");
  NECTB_REQUIRE(!(phase & kPhaseBackward) || (grid_grad && mlp_grad), "null gradient buffers");
  NECTB_REQUIRE(phase != (kPhaseForward | kPhaseBackward) || loss, "null loss");
  NECTB_REQUIRE(sub >= 1 && sub <= kMaxSubAngles, "sub_angles must be 1..%d (got %d)", kMaxSubAngles, sub);
  NECTB_REQUIRE(sub == 1 || sub_angles, "null sub-angle array");
  NECTB_REQUIRE((int64_t)batch->num_rays * sub <= INT32_MAX, "num_rays * sub_angles exceeds 2^31 - 1");
  cudaStream_t s = (cudaStream_t)stream;
  if (loss)
    if (int rc = cuda_status(cudaMemsetAsync(loss, 0, sizeof(float), s), "memset loss")) return rc;
  if (batch->num_rays == 0) return NECTB_OK;  // per-ray arrays may be null
  NECTB_REQUIRE(!(phase & kPhaseForward) || y_pred, "null y_pred");
  NECTB_REQUIRE(phase != kPhaseBackward || dloss_dy, "null dloss_dy");
  NECTB_REQUIRE(((uintptr_t)grid_grad & 15u) == 0 && ((uintptr_t)grid_params & 15u) == 0,
                "grid_grad and grid_params must be 16-byte aligned");
  NECTB_REQUIRE(batch->random_ray_index && batch->jitter && batch->detector_offset && batch->projection,
                "null batch input");
  const int P = geometry->nDetector[0] * geometry->nDetector[1];
  NECTB_REQUIRE((int64_t)P * sub <= INT32_MAX, "detector pixels * sub_angles exceeds 2^31 - 1");
  const int n_batch = batch->num_rays;
  const size_t need = sub > 1 ? scan_workspace_bytes(n_batch, P, sub) : workspace_bytes(n_batch, P);
  if (!workspace || workspace_size < need)
    return set_error(NECTB_ERR_WORKSPACE, "workspace of %zu bytes < required %zu", workspace_size, need);
  TrainArgs a;
  a.n_pixels = P * sub;
  a.perm = batch->random_ray_index;
  a.perm_len = batch->random_ray_index_len;
  a.start = batch->starting_ray_index;
  a.num_rays = n_batch * sub;
  a.S = batch->num_points_per_ray;
  a.angle = batch->angle_rad;
  a.t = batch->t;
  a.maxd = batch->max_ray_distance_per_point;
  a.uniform = batch->uniform_ray_spacing;
  a.max_dist = batch->max_distance_traveled;
  a.jitter = batch->jitter;
  a.det_off = batch->detector_offset;
  a.projection = batch->projection;
  a.loss_type = batch->loss_type;
  a.loss_scale = batch->loss_scale;
  a.max_blocks = 0;
  a.texture = texture;
  a.phase = phase;
  a.sub = sub;
  for (int j = 0; j < sub; ++j) a.sub_angle[j] = sub_angles ? sub_angles[j] : batch->angle_rad;
  Workspace ws = carve_workspace(workspace, a.num_rays, a.n_pixels, workspace_size);
  float* part = nullptr;  // continuous scan: each virtual ray's integral
  if (sub > 1) {
    part = reinterpret_cast<float*>(static_cast<char*>(workspace) + align256(workspace_bytes(a.num_rays, a.n_pixels)));
    const size_t pb = align256((size_t)a.num_rays * 4);
    if (ws.stage && ws.stage_bytes > pb) {
      ws.stage = reinterpret_cast<float*>(reinterpret_cast<char*>(ws.stage) + pb);
      ws.stage_bytes -= pb;
    } else {
      ws.stage = nullptr;
      ws.stage_bytes = 0;
    }
  }
  // the forward half has no loss output of its own: its loss sum lands in the workspace
  float* scratch_loss = reinterpret_cast<float*>(ws.counters + 8);
  float* fwd_loss = (sub > 1 || !loss) ? scratch_loss : loss;
  float* fwd_y = sub > 1 ? part : y_pred;
  if (phase & kPhaseForward) {
    if (int rc = cuda_status(cudaMemsetAsync(ws.counters, 0, 64, s), "memset counters")) return rc;
    if (int rc = cuda_status(cudaMemsetAsync(ws.slot, 0xFF, (size_t)a.n_pixels * 4, s), "memset slots")) return rc;
    ProfScope ps(kProfRayPrep, s);
    ray_prep_kernel<<<(unsigned)ceil_div(a.num_rays, 8), 256, 0, s>>>(*geometry, a, ws.rays, ws.slot, ws.counters,
                                                                       fwd_y, fwd_loss);
  } else {
    // backward half: fresh backward cursor, the caller's loss gradient per ray
    if (int rc = cuda_status(cudaMemsetAsync(ws.counters + 1, 0, sizeof(unsigned int), s), "memset cursor"))
      return rc;
    set_ray_grad_kernel<<<(unsigned)ceil_div(a.num_rays, 256), 256, 0, s>>>(ws.rays, dloss_dy, a.num_rays, n_batch,
                                                                            sub);
  }
  if (int rc = launch_status(phase & kPhaseForward ? "ray_prep_kernel" : "set_ray_grad_kernel")) return rc;
  const int nW = (int)mlp_param_count(mlp);
  const bool plain = mlp->compute_dtype == NECTB_F32;
  NECTB_REQUIRE(!plain || grid->feature_dtype == NECTB_F32, "plain path needs an fp32 table");
  auto run = [&](int ph, float* yp, float* ls) -> int {
    TrainArgs b = a;
    b.phase = ph;
    float* tg = (ph & kPhaseBackward) ? grid_grad : nullptr;
    float* mg = (ph & kPhaseBackward) ? mlp_grad : nullptr;
    if (plain) return train_plain(*geometry, g, *mlp, (const float*)grid_params, mlp_params, nW, b, ws, tg, mg, yp, ls, s);
    return train_mixed(*geometry, g, *mlp, grid_params, mlp_params, nW, b, ws, tg, mg, yp, ls, s);
  };
  if (sub == 1) return run(phase, y_pred, fwd_loss);
  // continuous scan: the forward kernels integrate every virtual ray, the
  // sub-angle average and the loss follow, then the backward
  if (phase & kPhaseForward) {
    if (int rc = run(kPhaseForward, part, scratch_loss)) return rc;
    scan_finalize_kernel<<<(unsigned)ceil_div(n_batch, 256), 256, 0, s>>>(
        ws.rays, part, n_batch, sub, y_pred, phase & kPhaseBackward ? loss : nullptr, a.loss_type, a.loss_scale,
        (phase & kPhaseBackward) ? 1 : 0);
    if (int rc = launch_status("scan_finalize_kernel")) return rc;
  }
  if (phase & kPhaseBackward) return run(kPhaseBackward, nullptr, nullptr);
  return NECTB_OK;
}

}  // namespace

// The fused training step with loads only: no texture object is made over
// the table (the allocation-free entry point creates no driver objects).
int train_step_loads_only(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                          const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                          float* grid_grad, float* mlp_grad, float* y_pred, float* loss, void* workspace,
                          size_t workspace_size, void* stream) {
  return train_entry(geometry, grid, mlp, grid_params, mlp_params, batch, nullptr, grid_grad, mlp_grad, y_pred, loss,
                     workspace, workspace_size, stream, kPhaseForward | kPhaseBackward, nullptr, 1, false);
}
}  // namespace nectb

extern "C" size_t nectb_train_scan_workspace_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                                   const NectbMLP* mlp, int32_t num_rays, int32_t sub_angles) {
  (void)grid;
  (void)mlp;
  const int P = geometry ? geometry->nDetector[0] * geometry->nDetector[1] : 0;
  return nectb::scan_workspace_bytes(std::max(num_rays, 1), std::max(P, 0), std::max(sub_angles, 1));
}

extern "C" int nectb_train_scan_step(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                                     const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                                     const float* sub_angles_rad, int32_t sub_angles, float* grid_grad,
                                     float* mlp_grad, float* y_pred, float* loss, void* workspace,
                                     size_t workspace_size, void* stream) {
  return nectb::train_entry(geometry, grid, mlp, grid_params, mlp_params, batch, nullptr, grid_grad, mlp_grad, y_pred,
                            loss, workspace, workspace_size, stream, nectb::kPhaseForward | nectb::kPhaseBackward,
                            sub_angles_rad, sub_angles);
}

extern "C" int nectb_train_scan_forward(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                                        const void* grid_params, const float* mlp_params,
                                        const NectbTrainBatch* batch, const float* sub_angles_rad, int32_t sub_angles,
                                        float* y_pred, void* workspace, size_t workspace_size, void* stream) {
  return nectb::train_entry(geometry, grid, mlp, grid_params, mlp_params, batch, nullptr, nullptr, nullptr, y_pred,
                            nullptr, workspace, workspace_size, stream, nectb::kPhaseForward, sub_angles_rad,
                            sub_angles);
}

extern "C" int nectb_train_scan_backward(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                         const NectbMLP* mlp, const void* grid_params, const float* mlp_params,
                                         const NectbTrainBatch* batch, const float* sub_angles_rad,
                                         int32_t sub_angles, const float* dloss_dy, float* grid_grad, float* mlp_grad,
                                         void* workspace, size_t workspace_size, void* stream) {
  return nectb::train_entry(geometry, grid, mlp, grid_params, mlp_params, batch, dloss_dy, grid_grad, mlp_grad,
                            nullptr, nullptr, workspace, workspace_size, stream, nectb::kPhaseBackward,
                            sub_angles_rad, sub_angles);
}

extern "C" const unsigned int* nectb_train_scan_error_word(const NectbGeometry* geometry, int32_t num_rays,
                                                           int32_t sub_angles, const void* workspace) {
  using namespace nectb;
  clear_error();
  if (!geometry || !workspace || num_rays <= 0 || sub_angles < 1 || sub_angles > kMaxSubAngles ||
      validate_geometry(geometry) != NECTB_OK) {
    set_error(NECTB_ERR_INVALID, "nectb_train_scan_error_word: invalid arguments");
    return nullptr;
  }
  const int P = geometry->nDetector[0] * geometry->nDetector[1];
  return carve_workspace(const_cast<void*>(workspace), num_rays * sub_angles, P * sub_angles).counters + 2;
}

extern "C" int nectb_train_step(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                                const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                                float* grid_grad, float* mlp_grad, float* y_pred, float* loss, void* workspace,
                                size_t workspace_size, void* stream) {
  return train_entry(geometry, grid, mlp, grid_params, mlp_params, batch, nullptr, grid_grad, mlp_grad, y_pred, loss,
                     workspace, workspace_size, stream, kPhaseForward | kPhaseBackward);
}

extern "C" int nectb_train_forward(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                                   const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                                   float* y_pred, void* workspace, size_t workspace_size, void* stream) {
  return train_entry(geometry, grid, mlp, grid_params, mlp_params, batch, nullptr, nullptr, nullptr, y_pred, nullptr,
                     workspace, workspace_size, stream, kPhaseForward);
}

extern "C" int nectb_train_backward(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                                    const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                                    const float* dloss_dy, float* grid_grad, float* mlp_grad, void* workspace,
                                    size_t workspace_size, void* stream) {
  return train_entry(geometry, grid, mlp, grid_params, mlp_params, batch, dloss_dy, grid_grad, mlp_grad, nullptr,
                     nullptr, workspace, workspace_size, stream, kPhaseBackward);
}

extern "C" int nectb_train_rays(const NectbGeometry* geometry, int32_t num_rays, int32_t num_points_per_ray,
                                const void* workspace, int32_t* counts, float* scale, float* points, void* stream) {
  using namespace nectb;
  clear_error();
  if (int rc = validate_geometry(geometry)) return rc;
  NECTB_REQUIRE(num_rays >= 0 && num_points_per_ray >= 1, "bad sizes");
  if (num_rays == 0) return NECTB_OK;
  NECTB_REQUIRE(workspace != nullptr, "null workspace");
  const int P = geometry->nDetector[0] * geometry->nDetector[1];
  const Workspace ws = carve_workspace(const_cast<void*>(workspace), num_rays, P);
  train_rays_kernel<<<(unsigned)ceil_div(num_rays, 8), 256, 0, (cudaStream_t)stream>>>(ws.rays, num_rays,
                                                                                        num_points_per_ray, counts,
                                                                                        scale, points);
  return launch_status("train_rays_kernel");
}

namespace nectb {
namespace {
// Recommended staging of the mixed path's two-pass backward for R (virtual)
// rays over P (virtual) pixels: ray order and offsets, the staged rounds, the
// encoding store (when enabled) and a 4D grid's time slice.
size_t staging_bytes(const NectbHashGrid* grid, int R, int P, int S) {
  const size_t per_ray = (size_t)S * grid->n_levels * grid->n_features * sizeof(float);
  const NectbTuning tune = current_tuning();
  const size_t row_bytes = (size_t)input_padded(grid->n_levels * grid->n_features) * 2;  // bf16 MLP input row
  const size_t rows = tune.encoding_store ? std::min<size_t>({(size_t)R * S, kEncodingStoreCap / row_bytes,
                                                             (size_t)0xffffffffu})
                                          : 0;
  size_t bytes = order_bytes(R, P) + staged_round_bytes(R, tune.staged_rounds, per_ray) + 256 +
                 align256(rows * row_bytes);
  GridDev g;
  if (tune.time_slice && grid->n_dims == 4 && make_grid_dev(grid, &g))
    bytes += slice_bytes(g) + 512;  // the time slice (512-byte aligned) and its gradient
  return bytes;
}
}  // namespace
}  // namespace nectb

extern "C" size_t nectb_train_staging_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                            const NectbMLP* mlp, int32_t num_rays, int32_t num_points_per_ray) {
  using namespace nectb;
  if (!geometry || !grid || !mlp || num_rays <= 0 || num_points_per_ray <= 0) return 0;
  if (mlp->compute_dtype == NECTB_F32) return 0;  // the plain path scatters in its backward
  return staging_bytes(grid, num_rays, geometry->nDetector[0] * geometry->nDetector[1], num_points_per_ray);
}

extern "C" size_t nectb_train_scan_staging_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                                 const NectbMLP* mlp, int32_t num_rays, int32_t num_points_per_ray,
                                                 int32_t sub_angles) {
  using namespace nectb;
  if (!geometry || !grid || !mlp || num_rays <= 0 || num_points_per_ray <= 0 || sub_angles < 1) return 0;
  if (mlp->compute_dtype == NECTB_F32) return 0;
  return staging_bytes(grid, num_rays * sub_angles, geometry->nDetector[0] * geometry->nDetector[1] * sub_angles,
                       num_points_per_ray);
}

namespace {
int model_backward_entry(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                         const float* mlp_params, const float* x, int64_t n, float t, const float* t_dev,
                         const float* dsigma, float* grid_grad, float* mlp_grad, void* stream) {
  clear_error();
  GridDev g;
  if (!make_grid_dev(grid, &g)) return set_error(NECTB_ERR_INVALID, "invalid hash grid description");
  if (int rc = validate_mlp(mlp, g)) return rc;
  NECTB_REQUIRE(n >= 0, "n must be >= 0");
  if (n == 0) return NECTB_OK;
  NECTB_REQUIRE(grid_params && mlp_params && x && dsigma && grid_grad && mlp_grad, "null pointer argument");
  NECTB_REQUIRE(((uintptr_t)grid_grad & 15u) == 0, "grid_grad must be 16-byte aligned");
  return model_backward(g, *mlp, grid->feature_dtype, grid_params, mlp_params, x, n, t, t_dev, dsigma, grid_grad,
                        mlp_grad, (cudaStream_t)stream);
}
}  // namespace

extern "C" int nectb_model_backward(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                                    const float* mlp_params, const float* x, int64_t n, float t, const float* dsigma,
                                    float* grid_grad, float* mlp_grad, void* stream) {
  return model_backward_entry(grid, mlp, grid_params, mlp_params, x, n, t, nullptr, dsigma, grid_grad, mlp_grad,
                              stream);
}

extern "C" int nectb_model_backward_t(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                                      const float* mlp_params, const float* x, int64_t n, const float* t,
                                      const float* dsigma, float* grid_grad, float* mlp_grad, void* stream) {
  if (!t) return set_error(NECTB_ERR_INVALID, "null timestep pointer");
  return model_backward_entry(grid, mlp, grid_params, mlp_params, x, n, 0.f, t, dsigma, grid_grad, mlp_grad,
                              stream);
}

extern "C" int nectb_adam_step(float* param, float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, double lr,
                               double beta1, double beta2, double eps, double weight_decay, int32_t step,
                               void* param_half, int32_t zero_grad, void* stream) {
  clear_error();
  if (n == 0) return NECTB_OK;
  NECTB_REQUIRE(param && grad && exp_avg && exp_avg_sq && n > 0 && step >= 1, "bad Adam arguments");
  const double bc1 = 1.0 - std::pow(beta1, step);
  const double bc2 = 1.0 - std::pow(beta2, step);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = (int)std::min<int64_t>(ceil_div(n, 256), (int64_t)sms * 8);
  const AdamScalars c{(float)(1.0 - beta1), (float)beta2, (float)(1.0 - beta2), (float)eps, (float)weight_decay,
                      (float)(-lr / bc1), (float)std::sqrt(bc2)};
  auto a16 = [](const void* q) { return ((uintptr_t)q & 15u) == 0; };
  const int vec = a16(param) && a16(grad) && a16(exp_avg) && a16(exp_avg_sq) && (((uintptr_t)param_half & 7u) == 0);
  ProfScope ps(kProfAdam, (cudaStream_t)stream);
  adam_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(param, grad, exp_avg, exp_avg_sq, n, c, (__half*)param_half,
                                                        zero_grad, vec);
  return launch_status("adam_kernel");
}
