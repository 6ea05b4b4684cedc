// Plain fp32 fused training step (SIMT MLP), the path the mixed-precision
// tensor-core kernels are measured against.
//
// Three launches per batch:
//   1. ray_prep_kernel   warp per ray: entry/exit, count, measured value.
//   2. fwd_plain_kernel  warp per ray: regenerate each sample, encode, MLP,
//                        warp-shuffle sum along the ray -> y_pred, loss,
//                        dL/dsigma for the ray.
//   3. bwd_plain_kernel  blocks of NT threads step through tiles of NT
//                        samples: re-encode, forward, backward through the
//                        MLP, fp32 weight-gradient tile products accumulated
//                        in registers, table gradients by float2/float4
//                        atomics.
// Sample positions and encodings live only in registers and shared memory.
#include <algorithm>

#include "mlp_simt.cuh"
#include "train_common.cuh"

namespace nectb {

__global__ void ray_prep_kernel(NectbGeometry g, TrainArgs a, RayRec* __restrict__ recs, int32_t* __restrict__ slot,
                                unsigned int* __restrict__ ctrl, float* __restrict__ y_pred, float* __restrict__ loss) {
  const int lane = threadIdx.x & 31;
  const int tid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (tid >= a.num_rays) return;
  int ray_index = 0;
  RaySetup r;
  r.valid = 0;
  r.distance = 0.f;
  // continuous scan: virtual ray tid is pixel rb of the batch at sub-angle j
  const int n_batch = a.num_rays / a.sub;
  const int j = tid / n_batch, rb = tid - j * n_batch;
  const float angle = a.sub > 1 ? a.sub_angle[j] : a.angle;
  // perm == nullptr: the detector pixels start, start + 1, ... in order
  // (re-projection queries, whole views or pieces of them; the slots are
  // indexed from the first pixel); jitter / detector offsets default to 0
  // when absent.
  bool ok;
  int sidx;  // scheduling slot of the ray's pixel
  if (a.perm) {
    ok = ray_lookup(a.perm, a.perm_len, a.start, rb, n_batch, g, ray_index);
    sidx = ray_index;
  } else {
    ray_index = (int)a.start + tid;
    ok = tid < a.n_pixels;
    sidx = tid;
  }
  if (ok)
    ray_setup(g, ray_index, a.det_off ? a.det_off[2 * (int64_t)tid] : 0.f,
              a.det_off ? a.det_off[2 * (int64_t)tid + 1] : 0.f, a.jitter ? a.jitter[tid] : 0.f, angle, a.S,
              a.maxd, a.uniform != 0, r);
  int count = 0;
  if (r.valid) count = warp_sample_count(g, r, a.S, lane);
  if (lane == 0) {
    RayRec rec;
    rec.sx = r.start.x;
    rec.sy = r.start.y;
    rec.sz = r.start.z;
    rec.dx = r.step.x;
    rec.dy = r.step.y;
    rec.dz = r.step.z;
    rec.count = count;
    rec.scale = r.distance / a.max_dist;
    // proj[perm[start:start+R]] (projector.py:130); rays past the end of the
    // permutation are not part of the reference batch and get y = 0 here.
    const bool in_range = ok && ray_index >= 0;
    rec.y = (in_range && a.projection) ? a.projection[ray_index] : 0.f;
    rec.gsig = 0.f;
    if (count > 0) {
      if (atomicCAS(slot + (int64_t)sidx * a.sub + j, -1, tid) != -1) atomicOr(ctrl + 3, kFlagDuplicatePixels);
    } else {
      // no samples: y_pred = 0 (the reference's zero attenuation sum)
      y_pred[tid] = 0.f;
      rec.gsig = loss_grad(0.f, rec.y, a.loss_type, a.num_rays, rec.scale) * a.loss_scale;
      atomicAdd(loss, loss_term(0.f, rec.y, a.loss_type) / (float)a.num_rays);
    }
    recs[tid] = rec;
  }
}

__device__ __forceinline__ bool ordered_valid(const int32_t* __restrict__ slot, const RayRec* __restrict__ recs,
                                              bool by_pixel, int idx, int n, int* ray) {
  if (idx >= n) return false;
  const int r = by_pixel ? slot[idx] : idx;
  *ray = r;
  return r >= 0 && recs[r].count > 0;
}

// Exclusive scan of one value per thread over a block of kOrderBlock threads
// (32 warps); returns the thread's prefix, *total the block's sum.  Callers
// that scan again into the same warp_sums synchronise first.
template <typename T>
__device__ __forceinline__ T block_scan(T v, T* warp_sums, T* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const T w = warp_sums[lane];
    T z = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += y;
    }
    warp_sums[lane] = z - w;  // exclusive over warps
    if (lane == 31) warp_sums[32] = z;
  }
  __syncthreads();
  *total = warp_sums[32];
  return warp_sums[warp] + x - v;
}

__global__ void __launch_bounds__(kOrderBlock)
order_count_kernel(const int32_t* __restrict__ slot, const RayRec* __restrict__ recs,
                   const unsigned int* __restrict__ ctrl, int R, int P, unsigned int* __restrict__ block_sums,
                   unsigned long long* __restrict__ block_samples) {
  __shared__ unsigned int ws[33];
  __shared__ unsigned long long ws64[33];
  const bool by_pixel = !(ctrl[3] & kFlagDuplicatePixels);
  int ray = -1;
  const bool v = ordered_valid(slot, recs, by_pixel, blockIdx.x * kOrderBlock + threadIdx.x, by_pixel ? P : R, &ray);
  unsigned int total;
  unsigned long long samples;
  block_scan<unsigned int>(v ? 1u : 0u, ws, &total);
  block_scan<unsigned long long>(v ? (unsigned long long)recs[ray].count : 0ull, ws64, &samples);
  if (threadIdx.x == 0) {
    block_sums[blockIdx.x] = total;
    block_samples[blockIdx.x] = samples;
  }
}

__global__ void __launch_bounds__(kOrderBlock)
order_scan_kernel(unsigned int* __restrict__ block_sums, unsigned long long* __restrict__ block_samples, int n_blocks,
                  unsigned int* __restrict__ ctrl) {
  __shared__ unsigned int ws[33];
  __shared__ unsigned long long ws64[33];
  unsigned int carry = 0;
  unsigned long long carry64 = 0;
  for (int b0 = 0; b0 < n_blocks; b0 += kOrderBlock) {  // block-uniform loop
    const int b = b0 + threadIdx.x;
    unsigned int total;
    unsigned long long total64;
    const unsigned int x = block_scan<unsigned int>(b < n_blocks ? block_sums[b] : 0u, ws, &total);
    const unsigned long long x64 = block_scan<unsigned long long>(b < n_blocks ? block_samples[b] : 0ull, ws64,
                                                                  &total64);
    if (b < n_blocks) {
      block_sums[b] = carry + x;
      block_samples[b] = carry64 + x64;
    }
    carry += total;
    carry64 += total64;
    __syncthreads();
  }
  if (threadIdx.x == 0) ctrl[6] = carry;  // rays with samples
}

__global__ void __launch_bounds__(kOrderBlock)
order_compact_kernel(const int32_t* __restrict__ slot, const RayRec* __restrict__ recs,
                     const unsigned int* __restrict__ ctrl, int R, int P, const unsigned int* __restrict__ block_sums,
                     const unsigned long long* __restrict__ block_samples, int32_t* __restrict__ order,
                     uint64_t* __restrict__ offs) {
  __shared__ unsigned int ws[33];
  __shared__ unsigned long long ws64[33];
  const bool by_pixel = !(ctrl[3] & kFlagDuplicatePixels);
  int ray = -1;
  const bool v = ordered_valid(slot, recs, by_pixel, blockIdx.x * kOrderBlock + threadIdx.x, by_pixel ? P : R, &ray);
  unsigned int total;
  unsigned long long samples;
  const unsigned int rank = block_scan<unsigned int>(v ? 1u : 0u, ws, &total);
  const unsigned long long off =
      block_scan<unsigned long long>(v ? (unsigned long long)recs[ray].count : 0ull, ws64, &samples);
  if (v) {
    order[block_sums[blockIdx.x] + rank] = ray;
    offs[block_sums[blockIdx.x] + rank] = block_samples[blockIdx.x] + off;
  }
}

namespace {

constexpr int kPlainFwdThreads = 128;

template <int D, int F, int IN, int H>
__global__ void __launch_bounds__(kPlainFwdThreads)
fwd_plain_kernel(GridDev grid, const float* __restrict__ table, const float* __restrict__ W, TrainArgs a,
                 RayRec* __restrict__ recs, const int32_t* __restrict__ slot, unsigned int* __restrict__ ctrl,
                 int act, int out_act, float* __restrict__ y_pred, float* __restrict__ loss) {
  constexpr int NT = kPlainFwdThreads;
  const bool by_pixel = !(ctrl[3] & kFlagDuplicatePixels);
  constexpr int LD = NT + 4;
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const SimtWeights sw = stage_weights<IN, H, false>(W, smem);
  float* cols = smem + simt_weight_floats<IN, H, false>();
  const int t = threadIdx.x;
  float* x = cols + t;                 // [IN][LD]
  float* hid = cols + IN * LD + t;     // two [64][LD] buffers, alternating between layers
  __syncthreads();
  const int lane = t & 31;
  float loss_acc = 0.f;
  while (true) {
    const int r = next_ray(ctrl, slot, recs, a.num_rays, a.n_pixels, by_pixel, lane);
    if (r < 0) break;
    const RayRec rec = load_ray(recs, r);
    float sum = 0.f;
    for (int base = 0; base < rec.count; base += 32) {
      const int i = base + lane;
      float p[4] = {0.f, 0.f, 0.f, 0.f};
      bool valid = false;
      if (i < rec.count) valid = sample_point(rec, i, p);
      if (D == 4) p[3] = a.t;
      if (valid) {
        encode_point<D, F, float>(grid, table, p, x, LD);
        const float* in = x;
        if (H == 1) {
          sum += act_fwd(gemv_dot<IN, LD>(sw.WT[0], in, sw.wout, act), out_act);
        } else {
          gemv_cols<IN, kWidth, LD>(sw.WT[0], in, hid, act);
#pragma unroll
          for (int k = 1; k < H - 1; ++k)
            gemv_cols<kWidth, kWidth, LD>(sw.WT[k], hid + ((k - 1) & 1) * kWidth * LD, hid + (k & 1) * kWidth * LD,
                                          act);
          sum += act_fwd(gemv_dot<kWidth, LD>(sw.WT[H - 1], hid + ((H - 2) & 1) * kWidth * LD, sw.wout, act),
                         out_act);
        }
      }
    }
    sum = warp_sum(sum);
    if (lane == 0) {
      const float yp = sum * rec.scale;
      y_pred[r] = yp;
      recs[r].gsig = loss_grad(yp, rec.y, a.loss_type, a.num_rays, rec.scale) * a.loss_scale;
      loss_acc += loss_term(yp, rec.y, a.loss_type);
    }
  }
  __shared__ float red[NT / 32];
  if (lane == 0) red[t >> 5] = loss_acc;
  __syncthreads();
  if (t == 0) {
    float s = 0.f;
    for (int w = 0; w < NT / 32; ++w) s += red[w];
    atomicAdd(loss, s / (float)a.num_rays);
  }
}

// acc[a][b] += sum_t G[(4*jb + a)*LD + t] * A[(ib*IB + b)*LD + t] over the
// tile's NT samples (weight gradient dW[j][i] = sum_t G[t][j] A[t][i]).
// Thread p owns rows 4*jb..4*jb+3 and columns ib*IB..ib*IB+IB-1.
template <int K, int NT, int LD>
struct WGrad {
  static constexpr int IBLK = NT / 16;
  static constexpr int IB = K / IBLK;
  static_assert(16 * IBLK == NT && IB * IBLK == K, "tile shape");
  float acc[4][IB];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < IB; ++b) acc[a][b] = 0.f;
  }
  __device__ __forceinline__ void add(const float* __restrict__ G, const float* __restrict__ A) {
    const int jb = threadIdx.x / IBLK, ib = threadIdx.x % IBLK;
#pragma unroll 1
    for (int t = 0; t < NT; t += 4) {
      float4 g[4], v[IB];
#pragma unroll
      for (int a = 0; a < 4; ++a) g[a] = *reinterpret_cast<const float4*>(G + (4 * jb + a) * LD + t);
#pragma unroll
      for (int b = 0; b < IB; ++b) v[b] = *reinterpret_cast<const float4*>(A + (ib * IB + b) * LD + t);
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < IB; ++b) {
          acc[a][b] = fmaf(g[a].x, v[b].x, acc[a][b]);
          acc[a][b] = fmaf(g[a].y, v[b].y, acc[a][b]);
          acc[a][b] = fmaf(g[a].z, v[b].z, acc[a][b]);
          acc[a][b] = fmaf(g[a].w, v[b].w, acc[a][b]);
        }
    }
  }
  __device__ __forceinline__ void flush(float* __restrict__ dst) const {  // dst [64][K]
    const int jb = threadIdx.x / IBLK, ib = threadIdx.x % IBLK;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < IB; ++b) atomicAdd(dst + (4 * jb + a) * K + ib * IB + b, acc[a][b]);
  }
};

// Whether the layer-0 weight-gradient tile stays in registers across the
// sample-tile loop.  A thread carries 4 * (IN + (H - 1) * 64) / (NT / 16)
// accumulators when every tile stays; the 3-layer MLP over 64 inputs (192 of
// them, the kernel at the 255-register limit) measured wrong first-layer and
// table gradients on B200 in that form, and exact ones when its layer-0 tile
// is added to W_grad after every sample tile (4096 atomics per tile of NT
// samples, about 64 per sample) and only the hidden-layer tiles stay.
template <int IN, int H, int NT>
__host__ __device__ constexpr bool carry_layer0() {
  return 4 * (IN + (H - 1) * kWidth) / (NT / 16) <= 160;
}

// Whether the hidden layers' weight-gradient tiles stay in registers across
// the loop (at most 160 accumulators); otherwise each is computed and added
// to W_grad per sample tile, one layer at a time (the deep models).
template <int H, int NT>
__host__ __device__ constexpr bool carry_hidden() {
  return 4 * (H - 1) * kWidth / (NT / 16) <= 160;
}

// Shared-memory plan of the SIMT backward kernels for IN inputs and H hidden
// layers: tiles of 128, 64 or 32 samples with both weight copies in shared
// memory, or, when even 32 do not fit (the deep models), tiles of 32 with the
// PyTorch-layout weights read from the global buffer through L1.
template <int IN, int H>
struct SimtBwdPlan {
  static constexpr size_t kBudget = 227 * 1024;
  static constexpr size_t cols(int nt) { return (size_t)(IN + (H + 2) * kWidth) * (nt + 4) * 4; }
  static constexpr size_t wbytes(bool both) {
    return (size_t)(both ? simt_weight_floats<IN, H, true>() : simt_weight_floats<IN, H, false>()) * 4;
  }
  static constexpr bool kBoth = wbytes(true) + cols(32) <= kBudget;
  static constexpr int NT =
      wbytes(kBoth) + cols(128) <= kBudget ? 128 : (wbytes(kBoth) + cols(64) <= kBudget ? 64 : 32);
  static constexpr size_t smem = wbytes(kBoth) + cols(NT);
  static_assert(smem <= kBudget, "SIMT backward does not fit shared memory");
};

template <int D, int F, int IN, int H, int NT, bool kBoth>
__global__ void __launch_bounds__(NT, 1)
bwd_plain_kernel(GridDev grid, const float* __restrict__ table, const float* __restrict__ W, TrainArgs a,
                 const RayRec* __restrict__ recs, const int32_t* __restrict__ slot, unsigned int* __restrict__ ctrl,
                 int act, int out_act, float* __restrict__ table_grad, float* __restrict__ W_grad) {
  constexpr int NW = NT / 32;
  const bool by_pixel = !(ctrl[3] & kFlagDuplicatePixels);
  constexpr int LD = NT + 4;
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const SimtWeights sw = stage_weights<IN, H, kBoth>(W, smem);
  float* cols = smem + simt_weight_floats<IN, H, kBoth>();
  float* sX = cols;                      // [IN][LD]
  float* sA = sX + IN * LD;              // [H][64][LD]  a_1..a_H
  float* sG = sA + H * kWidth * LD;      // [64][LD]
  float* sG2 = sG + kWidth * LD;         // [64][LD]
  const int t = threadIdx.x;
  const int lane = t & 31;
  (void)NW;
  constexpr bool kCarry0 = carry_layer0<IN, H, NT>();
  constexpr bool kCarryH = carry_hidden<H, NT>();
  WGrad<IN, NT, LD> g0;
  g0.zero();
  WGrad<kWidth, NT, LD> gh[kCarryH && H > 1 ? H - 1 : 1];
#pragma unroll
  for (int k = 0; k < (kCarryH ? H - 1 : 1); ++k) gh[k].zero();
  float dwout[2] = {0.f, 0.f};  // lane owns w_out[lane] and w_out[lane + 32]

  int ray = -1, base = 0;
  RayRec rec;
  rec.count = 0;
  rec.gsig = 0.f;
  __syncthreads();
  while (true) {
    if (ray < a.num_rays && (ray < 0 || base >= rec.count)) {
      const int r = next_ray(ctrl + 1, slot, recs, a.num_rays, a.n_pixels, by_pixel, lane);
      if (r < 0) {
        ray = a.num_rays;
        rec.count = 0;
      } else {
        rec = load_ray(recs, r);
        ray = r;
        base = 0;
      }
    }
    const bool warp_active = ray < a.num_rays;
    if (!__syncthreads_or(warp_active)) break;

    const int i = base + lane;
    float p[4] = {0.f, 0.f, 0.f, 0.f};
    bool valid = false;
    if (warp_active && i < rec.count) valid = sample_point(rec, i, p);
    if (D == 4) p[3] = a.t;
    if (valid) {
      encode_point<D, F, float>(grid, table, p, sX + t, LD);
    } else {
      for (int k = 0; k < IN; ++k) sX[k * LD + t] = 0.f;
    }
    // forward: a_1..a_H into sA
    gemv_cols<IN, kWidth, LD>(sw.WT[0], sX + t, sA + t, act);
#pragma unroll
    for (int k = 1; k < H; ++k)
      gemv_cols<kWidth, kWidth, LD>(sw.WT[k], sA + (k - 1) * kWidth * LD + t, sA + k * kWidth * LD + t, act);
    const float* aH = sA + (H - 1) * kWidth * LD + t;
    const float z = dot_col<kWidth, LD>(sw.wout, aH);
    const float dz = valid ? rec.gsig * act_grad_z(z, out_act) : 0.f;
    // w_out gradient (sum over the warp's samples), and G_H = dz * w_out * act'(a_H)
#pragma unroll 4
    for (int j = 0; j < kWidth; ++j) {
      const float aj = aH[j * LD];
      const float v = warp_sum(dz * aj);
      if ((j & 31) == lane) dwout[j >> 5] += v;
      sG[j * LD + t] = dz * sw.wout[j] * act_grad_a(aj, act);
    }
    float* G = sG;
    float* G2 = sG2;
#pragma unroll
    for (int k = H - 1; k >= 1; --k) {
      __syncthreads();
      if constexpr (kCarryH) {
        gh[k - 1].add(G, sA + (k - 1) * kWidth * LD);
      } else {  // this layer's tile, added to W_grad now
        gh[0].zero();
        gh[0].add(G, sA + (k - 1) * kWidth * LD);
        gh[0].flush(W_grad + kWidth * IN + (k - 1) * kWidth * kWidth);
      }
      // G_k = (W_k^T G_{k+1}) * act'(a_k); W_k is [64 out][64 in] = M[j][i]
      gemv_cols<kWidth, kWidth, LD>(sw.W[k], G + t, G2 + t, NECTB_ACT_NONE);
      const float* ak = sA + (k - 1) * kWidth * LD + t;
      for (int j = 0; j < kWidth; ++j) G2[j * LD + t] *= act_grad_a(ak[j * LD], act);
      float* tmp = G;
      G = G2;
      G2 = tmp;
    }
    __syncthreads();
    if constexpr (!kCarry0) g0.zero();
    g0.add(G, sX);
    if constexpr (!kCarry0) g0.flush(W_grad);
    // dX = W_0^T G_1 (W_0 is [64][IN] = M[j][i]) into G2, then scatter
    gemv_cols<kWidth, IN, LD>(sw.W[0], G + t, G2 + t, NECTB_ACT_NONE);
    // per-sample atomics: the SIMT path is issue-bound and the run reduction's
    // shuffles cost it more than the atomics they save (measured)
    scatter_warp<D, F>(grid, table_grad, p, valid, G2 + t, (int64_t)F * LD, LD, 0u, 0, grid.n_levels);
    __syncthreads();
    base += 32;
  }
  if constexpr (kCarry0) g0.flush(W_grad);
  if constexpr (kCarryH) {
#pragma unroll
    for (int k = 0; k < H - 1; ++k) gh[k].flush(W_grad + kWidth * IN + k * kWidth * kWidth);
  }
  const int nHidden = kWidth * IN + (H - 1) * kWidth * kWidth;
  // combine the warps' w_out partials through shared memory (reuse sG)
  __syncthreads();
  float* red = sG;  // [NW][64]
  red[(t >> 5) * kWidth + lane] = dwout[0];
  red[(t >> 5) * kWidth + lane + 32] = dwout[1];
  __syncthreads();
  for (int j = t; j < kWidth; j += NT) {  // tiles of 32 samples: each thread adds two entries
    float s = 0.f;
    for (int w = 0; w < NT / 32; ++w) s += red[w * kWidth + j];
    atomicAdd(W_grad + nHidden + j, s);
  }
}

// Backward of the model at n independent points (nectb_model_backward):
// gradients of sum_i dsigma[i] * sigma(x_i) added to the table and weight
// gradients.  The pipeline of bwd_plain_kernel (fp32 SIMT MLP, register tile
// weight gradients, per-sample table reductions) with points read from x
// (n x 3, (z, y, x); t broadcast in 4D) instead of regenerated along rays
// and a per-point dL/dsigma.  Tables of either precision are gathered.
template <int D, int F, int IN, int H, int NT, bool kBoth, typename T>
__global__ void __launch_bounds__(NT, 1)
model_bwd_kernel(GridDev grid, const T* __restrict__ table, const float* __restrict__ W, const float* __restrict__ x,
                 int64_t n, float tval, const float* __restrict__ t_dev, const float* __restrict__ dsigma, int act,
                 int out_act, float* __restrict__ table_grad, float* __restrict__ W_grad) {
  constexpr int LD = NT + 4;
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const SimtWeights sw = stage_weights<IN, H, kBoth>(W, smem);
  float* cols = smem + simt_weight_floats<IN, H, kBoth>();
  float* sX = cols;                      // [IN][LD]
  float* sA = sX + IN * LD;              // [H][64][LD]
  float* sG = sA + H * kWidth * LD;      // [64][LD]
  float* sG2 = sG + kWidth * LD;         // [64][LD]
  const int t = threadIdx.x;
  const int lane = t & 31;
  constexpr bool kCarry0 = carry_layer0<IN, H, NT>();
  constexpr bool kCarryH = carry_hidden<H, NT>();
  WGrad<IN, NT, LD> g0;
  g0.zero();
  WGrad<kWidth, NT, LD> gh[kCarryH && H > 1 ? H - 1 : 1];
#pragma unroll
  for (int k = 0; k < (kCarryH ? H - 1 : 1); ++k) gh[k].zero();
  float dwout[2] = {0.f, 0.f};
  if (D == 4 && t_dev) tval = *t_dev;   // the broadcast timestep, read on the device
  __syncthreads();
  for (int64_t c0 = (int64_t)blockIdx.x * NT; c0 < n; c0 += (int64_t)gridDim.x * NT) {  // block-uniform
    const int64_t i = c0 + t;
    const bool valid = i < n;
    float p[4] = {0.f, 0.f, 0.f, 0.f};
    if (valid) {
#pragma unroll
      for (int k = 0; k < 3; ++k) p[k] = x[i * 3 + k];
    }
    if (D == 4) p[3] = tval;
    if (valid) {
      encode_point<D, F, T>(grid, table, p, sX + t, LD);
    } else {
      for (int k = 0; k < IN; ++k) sX[k * LD + t] = 0.f;
    }
    gemv_cols<IN, kWidth, LD>(sw.WT[0], sX + t, sA + t, act);
#pragma unroll
    for (int k = 1; k < H; ++k)
      gemv_cols<kWidth, kWidth, LD>(sw.WT[k], sA + (k - 1) * kWidth * LD + t, sA + k * kWidth * LD + t, act);
    const float* aH = sA + (H - 1) * kWidth * LD + t;
    const float z = dot_col<kWidth, LD>(sw.wout, aH);
    const float dz = valid ? dsigma[i] * act_grad_z(z, out_act) : 0.f;
#pragma unroll 4
    for (int j = 0; j < kWidth; ++j) {
      const float aj = aH[j * LD];
      const float v = warp_sum(dz * aj);
      if ((j & 31) == lane) dwout[j >> 5] += v;
      sG[j * LD + t] = dz * sw.wout[j] * act_grad_a(aj, act);
    }
    float* G = sG;
    float* G2 = sG2;
#pragma unroll
    for (int k = H - 1; k >= 1; --k) {
      __syncthreads();
      if constexpr (kCarryH) {
        gh[k - 1].add(G, sA + (k - 1) * kWidth * LD);
      } else {  // this layer's tile, added to W_grad now
        gh[0].zero();
        gh[0].add(G, sA + (k - 1) * kWidth * LD);
        gh[0].flush(W_grad + kWidth * IN + (k - 1) * kWidth * kWidth);
      }
      gemv_cols<kWidth, kWidth, LD>(sw.W[k], G + t, G2 + t, NECTB_ACT_NONE);
      const float* ak = sA + (k - 1) * kWidth * LD + t;
      for (int j = 0; j < kWidth; ++j) G2[j * LD + t] *= act_grad_a(ak[j * LD], act);
      float* tmp = G;
      G = G2;
      G2 = tmp;
    }
    __syncthreads();
    if constexpr (!kCarry0) g0.zero();
    g0.add(G, sX);
    if constexpr (!kCarry0) g0.flush(W_grad);
    gemv_cols<kWidth, IN, LD>(sw.W[0], G + t, G2 + t, NECTB_ACT_NONE);
    scatter_warp<D, F>(grid, table_grad, p, valid, G2 + t, (int64_t)F * LD, LD, 0u, 0, grid.n_levels);
    __syncthreads();
  }
  if constexpr (kCarry0) g0.flush(W_grad);
  if constexpr (kCarryH) {
#pragma unroll
    for (int k = 0; k < H - 1; ++k) gh[k].flush(W_grad + kWidth * IN + k * kWidth * kWidth);
  }
  const int nHidden = kWidth * IN + (H - 1) * kWidth * kWidth;
  __syncthreads();
  float* red = sG;  // [NT/32][64]
  red[(t >> 5) * kWidth + lane] = dwout[0];
  red[(t >> 5) * kWidth + lane + 32] = dwout[1];
  __syncthreads();
  for (int j = t; j < kWidth; j += NT) {  // tiles of 32 samples: each thread adds two entries
    float s = 0.f;
    for (int w = 0; w < NT / 32; ++w) s += red[w * kWidth + j];
    atomicAdd(W_grad + nHidden + j, s);
  }
}

template <int D, int F, int L, int H, typename T>
int launch_model_bwd(const GridDev& grid, const void* table, const float* W, const float* x, int64_t n, float tval,
                     const float* t_dev, const float* dsigma, int act, int out_act, float* table_grad, float* W_grad,
                     cudaStream_t s) {
  constexpr int IN = L * F;
  using Plan = SimtBwdPlan<IN, H>;
  constexpr int NT = Plan::NT;
  auto k = model_bwd_kernel<D, F, IN, H, NT, Plan::kBoth, T>;
  const size_t smem = Plan::smem;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(sms, ceil_div(n, NT)));
  ProfScope ps(kProfModel, s);
  k<<<blocks, NT, smem, s>>>(grid, (const T*)table, W, x, n, tval, t_dev, dsigma, act, out_act, table_grad, W_grad);
  return launch_status("model_bwd_kernel");
}

template <int D, int F, int L, int H>
int run_plain(const NectbGeometry& geo, const GridDev& grid, const float* table, const float* W, const TrainArgs& a,
              Workspace ws, int act, int out_act, float* table_grad, float* W_grad, float* y_pred, float* loss,
              cudaStream_t s) {
  constexpr int IN = L * F;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  (void)geo;

  constexpr int FNT = kPlainFwdThreads;
  auto fk = fwd_plain_kernel<D, F, IN, H>;
  const size_t fsmem =
      (size_t)(simt_weight_floats<IN, H, false>() + (IN + simt_hidden_buffers<H>() * kWidth) * (FNT + 4)) * 4;
  set_smem(fk, fsmem, a.max_blocks > 0);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fk, FNT, fsmem);
  int fblocks = std::max(1, std::min<int>(sms * std::max(per_sm, 1), (int)ceil_div(a.num_rays, FNT / 32)));
  if (a.max_blocks > 0) fblocks = std::min(fblocks, a.max_blocks);
  if (a.phase & kPhaseForward) {
    {
      ProfScope ps(kProfForward, s);
      fk<<<fblocks, FNT, fsmem, s>>>(grid, table, W, a, ws.rays, ws.slot, ws.counters, act, out_act, y_pred, loss);
    }
    if (int rc = launch_status("fwd_plain_kernel")) return rc;
  }
  if (!table_grad || !(a.phase & kPhaseBackward)) return NECTB_OK;  // forward only (queries, split step)

  using Plan = SimtBwdPlan<IN, H>;
  constexpr int NT = Plan::NT;
  auto bk = bwd_plain_kernel<D, F, IN, H, NT, Plan::kBoth>;
  const size_t bsmem = Plan::smem;
  cudaFuncSetAttribute(bk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsmem);
  const int bblocks = std::max(1, std::min<int>(sms, (int)ceil_div(a.num_rays, NT / 32)));
  {
    ProfScope ps(kProfBackward, s);
    bk<<<bblocks, NT, bsmem, s>>>(grid, table, W, a, ws.rays, ws.slot, ws.counters, act, out_act, table_grad,
                                  W_grad);
  }
  return launch_status("bwd_plain_kernel");
}

}  // namespace

int model_backward(const GridDev& g, const NectbMLP& mlp, int dtype, const void* table, const float* W,
                   const float* x, int64_t n, float tval, const float* t_dev, const float* dsigma, float* table_grad,
                   float* W_grad, cudaStream_t s) {
  const bool h = dtype == NECTB_F16;
  const int D = g.n_dims, F = g.n_features, L = g.n_levels, H = mlp.n_hidden_layers;
  const int act = mlp.activation, oact = mlp.output_activation;
  const int rc = dispatch_shape(D, F, L, H, [&](auto d, auto f, auto l, auto hl) {
    return h ? launch_model_bwd<d(), f(), l(), hl(), __half>(g, table, W, x, n, tval, t_dev, dsigma, act, oact,
                                                             table_grad, W_grad, s)
             : launch_model_bwd<d(), f(), l(), hl(), float>(g, table, W, x, n, tval, t_dev, dsigma, act, oact,
                                                            table_grad, W_grad, s);
  });
  if (rc != kUnsupportedShape) return rc;
  return set_error(NECTB_ERR_INVALID, "model backward: unsupported configuration (n_dims %d, n_features %d, "
                   "n_levels %d, hidden %d)", D, F, L, H);
}

int train_plain(const NectbGeometry& geo, const GridDev& grid, const NectbMLP& mlp, const float* table,
                const float* W, int nW, const TrainArgs& a, Workspace ws, float* table_grad, float* W_grad,
                float* y_pred, float* loss, cudaStream_t s) {
  (void)nW;
  const int D = grid.n_dims, F = grid.n_features, L = grid.n_levels, H = mlp.n_hidden_layers;
  const int act = mlp.activation, oact = mlp.output_activation;
  const int rc = dispatch_shape(D, F, L, H, [&](auto d, auto f, auto l, auto h) {
    return run_plain<d(), f(), l(), h()>(geo, grid, table, W, a, ws, act, oact, table_grad, W_grad, y_pred, loss,
                                         s);
  });
  if (rc != kUnsupportedShape) return rc;
  return set_error(NECTB_ERR_INVALID, "plain path: unsupported model shape (n_dims %d, n_features %d, n_levels %d, "
                   "hidden %d)", D, F, L, H);
}

}  // namespace nectb
