// Mixed-precision fused training step: fp16 hash tables, bf16 MLP on the
// 5th-generation tensor cores (tcgen05.mma, fp32 accumulators in TMEM), fp32
// Kahan-compensated line integral, fp32 gradient tables.
//
// Block = 4 warps = one warpgroup; a tile is 128 samples (each warp 32
// consecutive samples of its current ray), i.e. the M = 128 rows of every
// MMA and the 128 TMEM lanes (warp w reads lanes 32w..32w+31 with
// tcgen05.ld.32x32b, so each thread owns its sample's row).  Per tile, with
// H hidden layers and hidden activation a():
//   forward:  X[128xIN] -> A1 = a(X W0^T) -> ... -> A_H = a(A_{H-1} W_{H-1}^T) -> sigma
//   backward: G_H = dsigma * w_out * a'(A_H)
//             dA_k = G_{k+1} W_k      dW_k += G_{k+1}^T A_k  (TMEM accumulator), k = H-1..1
//             G_k = dA_k * a'(A_k)
//             dX = G_1 W0             dW0 += G_1^T X          (TMEM accumulator)
//             table_grad[corner] += w_corner * dX   (fp32 vector reductions)
// Operands are 128-byte-swizzled bf16 tiles in shared memory; the same tile
// is the K-major A operand of the next layer and the MN-major operand of the
// weight-gradient product, so no transposed copies are made.  The weight
// gradients use M = 128 with the 64 real rows first (rows 64..127 read a
// second, unused tile and are never stored).  Inputs wider than 64 (the
// reference's default 19 x 4 levels) take two X tiles: layer 0 runs K over
// both, dX is an N = 128 product and the layer-0 weight gradient is taken
// transposed, dW0^T += X^T G_1, with the two X tiles as the M = 128 operand.
// One thread issues the MMAs and commits them to an mbarrier; every wait is
// bounded and reports through an error word instead of hanging.
#include <algorithm>
#include <mutex>
#include <tuple>
#include <vector>

#include "mixed_common.cuh"
#include "train_common.cuh"

namespace nectb {

namespace {

constexpr int kMixThreads = 128;
constexpr int kScatterThreads = 256;
// Per-warp ray cursor shared by the mixed kernels.
struct RayCursor {
  int ray = -1;
  int base = 0;
  int sched = 0;      // scheduling index (detector pixel, or batch position; rank with an order) of the ray
  int64_t xrow = -1;  // encoding-store row of the ray's sample 0, -1 if its rows are not stored
  RayRec rec;
};

// Advances the warp to its next chunk of 32 samples (a new ray from the
// scheduler when the current one is done).  Returns false when no rays are
// left.  Rays without samples were finalised by the preparation kernel.
// With ``order`` the rays come from the ordered list, ranks [lo, hi) (one
// round of the two-pass backward), else from the scheduling indices [lo, hi).
// With ``offs`` a ray whose rows all lie below xcap gets its store row.
__device__ __forceinline__ bool next_chunk(RayCursor& cur, const RayRec* recs, unsigned int* cursor,
                                           const int32_t* slot, const TrainArgs& a, bool by_pixel, int lane,
                                           int lo = 0, int hi = 0x7fffffff, const int32_t* order = nullptr,
                                           unsigned int n_valid = 0, const uint64_t* offs = nullptr,
                                           uint32_t xcap = 0) {
  if (cur.ray >= a.num_rays) return false;
  if (cur.ray >= 0 && cur.base < cur.rec.count) return true;
  const int r = order ? next_ray_ranked(cursor, order, n_valid, lo, hi, lane, &cur.sched)
                      : next_ray(cursor, slot, recs, a.num_rays, a.n_pixels, by_pixel, lane, lo, hi, &cur.sched);
  if (r < 0) {
    cur.ray = a.num_rays;
    cur.rec.count = 0;
    cur.xrow = -1;
    return false;
  }
  cur.rec = load_ray(recs, r);
  cur.ray = r;
  cur.base = 0;
  cur.xrow = -1;
  if (order && offs) {
    const uint64_t o = offs[cur.sched];
    if (o + (uint64_t)cur.rec.count <= (uint64_t)xcap) cur.xrow = (int64_t)o;
  }
  return true;
}

// Warpgroups of the forward per SM.  A block is one to kFwdBlocksPerSM
// independent warpgroups (128 threads each, one 128-sample tile, its own 64
// TMEM columns, mbarrier and named barrier) that share one copy of the weight
// tiles: with four, shared memory is 82 KB per SM instead of four blocks'
// 136 KB, and the L1 that the gathers hit (neighbouring rays reuse table
// entries) grows from 92 to 156 KB.  Every layer's product goes to the same
// 64 columns: the next layer's MMA is issued only after the warpgroup has
// read the previous result into registers, 32 columns at a time.  Six
// warpgroups (24 warps, 80 registers each) keep more gathers in flight than
// four (the forward is bound by gather latency and L1 throughput): C3
// forward 16.0 -> 14.6 ms.  Re-projection queries, which share SMs with
// serving kernels, run one warpgroup per block or the caller's number.
constexpr int kFwdBlocksPerSM = kFwdMaxWarpgroups;
static_assert(kFwdBlocksPerSM >= 1 && kFwdBlocksPerSM * 64 <= 512 && kFwdBlocksPerSM * 128 <= 1024,
              "TMEM holds 512 columns per SM, a block 1024 threads");
// The forward's warpgroups per SM for a model shape: all of them for 3D
// grids and two hidden layers (80 registers a thread suffice); deeper MLPs
// keep four and 128 registers (at 80 they would spill), and so do 4D grids:
// compiled for 80 registers the 4D forward's stored encoding rows disagreed
// with the recomputed ones (the staged backward's table gradient off by
// 4e-4 of its largest entry, the y_pred identical), while at 128 they agree
// bit for bit.  4D training runs the 3D kernels on the time slice.
template <int D, int L, int F, int H>
struct FwdShape {
  static constexpr int kMaxWarpgroups =
      (D == 3 && H == 2) ? kFwdBlocksPerSM : (kFwdBlocksPerSM < 4 ? kFwdBlocksPerSM : 4);
};

// TMEM columns of a forward block of n_wg warpgroups: 64 each, allocated as a power of two.
__host__ __device__ constexpr uint32_t fwd_tmem_cols(int n_wg) {
  return n_wg <= 1 ? 64u : (n_wg == 2 ? 128u : (n_wg <= 4 ? 256u : 512u));
}

// Barrier over the 128 threads of warpgroup wg (named barrier wg + 1; 0 is
// __syncthreads'), and its OR-reduction form.
__device__ __forceinline__ void wg_sync(int wg) { asm volatile("bar.sync %0, 128;" ::"r"(wg + 1) : "memory"); }
__device__ __forceinline__ bool wg_or(int wg, bool p) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, %2, 128, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)p), "r"(wg + 1)
      : "memory");
  return r != 0;
}

template <int D, int F, int L, int H, int ACT>
__global__ void __launch_bounds__(FwdShape<D, L, F, H>::kMaxWarpgroups * kMixThreads, 1)
fwd_mixed_kernel(GridDev grid, const __half* __restrict__ table, const float* __restrict__ W, TrainArgs a,
                 RayRec* __restrict__ recs, const int32_t* __restrict__ slot, unsigned int* __restrict__ ctrl,
                 int out_act, float* __restrict__ y_pred, float* __restrict__ loss,
                 const int32_t* __restrict__ order, const uint64_t* __restrict__ offs, uint4* __restrict__ xstore,
                 uint32_t xcap) {
  using S = InShape<L, F>;
  constexpr int KT = S::KT;
  constexpr int act = ACT;  // hidden activation, a compile-time constant of the hot loops
  const bool by_pixel = !(ctrl[3] & kFlagDuplicatePixels);
  const unsigned int n_valid = order ? ctrl[6] : 0u;
  unsigned int* err = ctrl + 2;
  const int n_wg = blockDim.x / kMixThreads;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = align1024(smem_raw);
  uint8_t* sW = base;  // KT + H - 1 weight tiles, shared by the warpgroups
  float* sWout = reinterpret_cast<float*>(sW + (KT + H - 1) * kWTile + n_wg * KT * kTile);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sWout + 64);       // [n_wg]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + kFwdBlocksPerSM);
  float* red = reinterpret_cast<float*>(tslot + 4);                 // [warps]

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int wg = t / kMixThreads, r = t % kMixThreads;  // warpgroup, and this thread's row of its tile
  // Each hidden layer's activations overwrite X (tile 0): the MMA that read the
  // tile has finished (its commit has arrived) before the next activations are
  // written, and the next X is written only after the last MMA has completed.
  uint8_t* sX = sW + (KT + H - 1) * kWTile + wg * KT * kTile;
  uint8_t* sA = sX;
  uint64_t* bar = bars + wg;
  if (xstore && blockIdx.x == 0 && t == 0) ctrl[7] = xcap;  // rows this forward fills, for the backward
  stage_mixed_weights<L, F, H>(W, sW, sWout);
  const uint32_t ncols = fwd_tmem_cols(n_wg);
  if (warp == 0) {
    tc::tmem_alloc(tslot, ncols);
    tc::tmem_relinquish();
  }
  if (r == 0) tc::mbar_init(bar, 1);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tm = *tslot + 64u * wg;  // this warpgroup's 64 columns
  const uint32_t my_lanes = tm + ((uint32_t)(32 * (warp & 3)) << 16);
  const uint32_t sX_a = tc::smem_u32(sX), sA_a = tc::smem_u32(sA), sW_a = tc::smem_u32(sW);
  constexpr uint32_t idesc = tc::idesc_bf16(128, 64, false, false);

  uint32_t phase = 0;
  float loss_acc = 0.f;
  float ksum = 0.f, kcomp = 0.f;  // Kahan sum of sigma along the warp's current ray (per lane)
  RayCursor cur;
  bool timed_out = false;
  while (true) {
    const bool active =
        next_chunk(cur, recs, ctrl, slot, a, by_pixel, lane, 0, 0x7fffffff, order, n_valid, offs, xcap);
    if (!wg_or(wg, active)) break;
    const int i = cur.base + lane;
    float p[4] = {0.f, 0.f, 0.f, 0.f};
    bool valid = false;
    if (active && i < cur.rec.count) valid = sample_point(cur.rec, i, p);
    if (D == 4) p[3] = a.t;
    encode_row<D, F, L>(grid, table, p, valid, sX, r,
                        valid && cur.xrow >= 0 ? xstore + (size_t)(cur.xrow + i) * S::NCH : nullptr);
    // layer k (0-based) writes the warpgroup's 64 TMEM columns; its input is
    // X for k = 0, else the previous layer's activations in sA (which
    // overwrite X once layer 0's MMA has completed)
    float z = 0.f;
#pragma unroll
    for (int k = 0; k < H; ++k) {
      tc::fence_async_smem();
      tc::fence_before();
      wg_sync(wg);
      if (r == 0) {
        tc::fence_after();
        if (k == 0) {
#pragma unroll
          for (int q = 0; q < S::INP / 16; ++q)
            tc::mma(tm, tc::desc_k(sX_a + (q / 4) * kTile, q % 4), tc::desc_k(sW_a + (q / 4) * kWTile, q % 4),
                    idesc, q > 0);
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            tc::mma(tm, tc::desc_k(sA_a, q), tc::desc_k(sW_a + (KT + k - 1) * kWTile, q), idesc, q > 0);
        }
        tc::commit(bar);
      }
      timed_out = !tc::mbar_wait(bar, phase);
      phase ^= 1;
      if (wg_or(wg, timed_out)) {
        timed_out = true;
        break;
      }
      tc::fence_after();
      // the layer's 64 values, 32 columns at a time: the hidden activations
      // into sA for the next layer, or the output layer's dot product
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        float v[32];
        tc::tmem_ld16(my_lanes + 32 * half, v);
        tc::tmem_ld16(my_lanes + 32 * half + 16, v + 16);
        tc::tmem_wait_ld();
        if (k + 1 < H) {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            float a8[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) a8[q] = hidden_act(v[8 * c + q], act);
            tc::st_chunk_bf16(sA, r, 4 * half + c, a8);
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j) z = fmaf(sWout[32 * half + j], hidden_act(v[j], act), z);
        }
      }
    }
    if (timed_out) break;
    if (valid) {  // Kahan-compensated accumulation along the ray
      const float y = act_fwd(z, out_act) - kcomp;
      const float s = ksum + y;
      kcomp = (s - ksum) - y;
      ksum = s;
    }
    tc::fence_before();
    if (active) {
      cur.base += 32;
      if (cur.base >= cur.rec.count) {
        const float sum = warp_sum(ksum);
        if (lane == 0) {
          const float yp = sum * cur.rec.scale;
          y_pred[cur.ray] = yp;
          recs[cur.ray].gsig = loss_grad(yp, cur.rec.y, a.loss_type, a.num_rays, cur.rec.scale) * a.loss_scale;
          loss_acc += loss_term(yp, cur.rec.y, a.loss_type);
        }
        ksum = 0.f;
        kcomp = 0.f;
      }
    }
  }
  if (timed_out && r == 0) atomicOr(err, 1u);
  if (lane == 0) red[warp] = loss_acc;
  tc::fence_before();
  __syncthreads();
  if (t == 0) {
    float sum = 0.f;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) sum += red[w];
    atomicAdd(loss, sum / (float)a.num_rays);
  }
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(*tslot, ncols);
  }
}

// Staged mode (kStaged): instead of scattering, dL/d(encoding) of every sample
// is written to the staging buffer, level-major: stage[(l * slots + s) * F + f]
// with s = (scheduling index - lo) * S + sample, for the rays whose
// scheduling index lies in [lo, hi); scatter_stage_kernel applies it.
//
// TMEM (BW columns): [0, T) the transient result of every layer and gradient
// product (T = 64, or 128 for the N = 128 dX of two X tiles), dW_k at
// T + 64 (k - 1) for k = 1..H-1, dW0 at T + 64 (H - 1): IN columns, or for
// two X tiles the transposed dW0^T, 64 columns in lanes 0..IN-1.
template <int L, int F, int H>
struct BwdPlan {
  using S = InShape<L, F>;
  static constexpr int T = S::KT == 2 ? 128 : 64;
  static constexpr int kUsed = T + 64 * H;
  static constexpr uint32_t kCols = kUsed <= 256 ? 256u : 512u;
  static_assert(kUsed <= 512, "TMEM plan exceeds 512 columns");
  static constexpr size_t smem = 1024 + (S::KT + H - 1) * kWTile + (H + S::KT) * kTile + 64 * 4 + 64 + 4 * 64 * 4;
};

template <int D, int F, int L, int H, bool kStaged, int ACT>
__global__ void __launch_bounds__(kMixThreads, 2)
bwd_mixed_kernel(GridDev grid, const __half* __restrict__ table, const float* __restrict__ W, TrainArgs a,
                 const RayRec* __restrict__ recs, const int32_t* __restrict__ slot, unsigned int* __restrict__ ctrl,
                 int out_act, float* __restrict__ table_grad, float* __restrict__ W_grad, int lo, int hi,
                 float* __restrict__ stage, int64_t slots, const int32_t* __restrict__ order,
                 const uint64_t* __restrict__ offs, const uint4* __restrict__ xstore, uint32_t xcap) {
  using S = InShape<L, F>;
  using Plan = BwdPlan<L, F, H>;
  constexpr int IN = S::IN, KT = S::KT;
  constexpr int act = ACT;
  static_assert(H >= 2, "at least two hidden layers");
  const bool by_pixel = !(ctrl[3] & kFlagDuplicatePixels);
  const unsigned int n_valid = order ? ctrl[6] : 0u;
  // rows below both this launch's store size and the forward's are valid
  const uint32_t xrows = xstore ? min(xcap, ctrl[7]) : 0u;
  unsigned int* err = ctrl + 2;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = align1024(smem_raw);
  // Tiles: sG (G_H), then A_{H-1} ... A_1 (each later replaced by G_k), then
  // the KT X tiles.  Order matters: the padded (M = 128) weight-gradient
  // products read a second 16 KB block right after their G tile, which is
  // always the next tile of this list, inside this block's allocation.
  uint8_t* sW = base;  // KT + H - 1 weight tiles
  uint8_t* sG = sW + (KT + H - 1) * kWTile;
  uint8_t* sX = sG + H * kTile;
  float* sWout = reinterpret_cast<float*>(sX + KT * kTile);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sWout + 64);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  float* red = reinterpret_cast<float*>(tslot + 4);  // [4][64]
  auto sAk = [&](int k) { return sG + (H - k) * kTile; };   // A_k (k = 1..H-1), later G_k

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  stage_mixed_weights<L, F, H>(W, sW, sWout);
  if (warp == 0) {
    tc::tmem_alloc(tslot, Plan::kCols);
    tc::tmem_relinquish();
  }
  if (t == 0) tc::mbar_init(bar, 1);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tm = *tslot;
  const uint32_t my_lanes = tm + ((uint32_t)(32 * warp) << 16);
  const uint32_t sX_a = tc::smem_u32(sX), sG_a = tc::smem_u32(sG), sW_a = tc::smem_u32(sW);
  const uint32_t dw0 = tm + Plan::T + 64 * (H - 1);
  // M = 128 weight-gradient products: rows 64..127 of A come from the tile kTile further on.
  const uint32_t pad_lbo = kTile;
  constexpr uint32_t id_fwd = tc::idesc_bf16(128, 64, false, false);
  constexpr uint32_t id_dA = tc::idesc_bf16(128, 64, false, true);
  constexpr uint32_t id_dW = tc::idesc_bf16(128, 64, true, true);
  constexpr uint32_t id_dX = tc::idesc_bf16(128, KT == 2 ? 128 : S::INP, false, true);
  constexpr uint32_t id_dW0 = tc::idesc_bf16(128, S::INP, true, true);

  uint32_t phase = 0;
  uint32_t wacc = 0;  // weight-gradient accumulators start at the first tile
  float dwout0 = 0.f, dwout1 = 0.f;  // w_out gradient entries j0_out and j0_out + 1 of this lane
  int j0_out = 0;
  RayCursor cur;
  bool timed_out = false;
  uint4 xrow[S::NCH];    // stored rows of the current chunk (this thread's sample)
  bool pre_ok = false;   // xrow already holds them (prefetched during the previous tile)
  // Issues the MMAs of one phase (thread 0), waits for them; false on time-out.
  auto run_phase = [&](auto issue) -> bool {
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    if (t == 0) {
      tc::fence_after();
      issue();
      tc::commit(bar);
    }
    const bool to = !tc::mbar_wait(bar, phase);
    phase ^= 1;
    if (__syncthreads_or(to)) return false;
    tc::fence_after();
    return true;
  };
  while (true) {
    const bool active =
        next_chunk(cur, recs, ctrl + 1, slot, a, by_pixel, lane, lo, hi, order, n_valid, offs, xrows);
    if (!__syncthreads_or(active)) break;
    const int i = cur.base + lane;
    float p[4] = {0.f, 0.f, 0.f, 0.f};
    bool valid = false;
    if (active && i < cur.rec.count) valid = sample_point(cur.rec, i, p);
    if (D == 4) p[3] = a.t;
    if (cur.xrow >= 0) {  // the forward stored this ray's rows: stream them back (warp-uniform branch)
      const uint4* src = xstore + (size_t)(cur.xrow + i) * S::NCH;
      if (!pre_ok && valid) {  // not prefetched: the first chunk of a ray
#pragma unroll
        for (int j = 0; j < S::NCH; ++j) xrow[j] = __ldcs(src + j);
      }
#pragma unroll
      for (int j = 0; j < S::NCH; ++j)
        tc::st_chunk_raw(sX + (j / 8) * kTile, t, j % 8, valid ? xrow[j] : make_uint4(0u, 0u, 0u, 0u));
      // prefetch the rows of the warp's next chunk of this ray; they arrive
      // while this tile's MMAs run (rows below the ray's count lie in its
      // stored range)
      pre_ok = cur.base + 32 < cur.rec.count;
      if (pre_ok && i + 32 < cur.rec.count) {
#pragma unroll
        for (int j = 0; j < S::NCH; ++j) xrow[j] = __ldcs(src + 32 * S::NCH + j);
      }
    } else {
      pre_ok = false;
      encode_row<D, F, L>(grid, table, p, valid, sX, t);
    }
    // forward recompute: layer 0 from X, layer k from A_k (stored with its sign mask)
    float h[64];
    uint32_t mlo[H], mhi[H];
    bool ok = run_phase([&] {
#pragma unroll
      for (int q = 0; q < S::INP / 16; ++q)
        tc::mma(tm, tc::desc_k(sX_a + (q / 4) * kTile, q % 4), tc::desc_k(sW_a + (q / 4) * kWTile, q % 4), id_fwd,
                q > 0);
    });
    if (ok) ld64(my_lanes, h);
#pragma unroll
    for (int k = 1; k < H && ok; ++k) {
      act_row(h, sAk(k), t, act, mlo[k], mhi[k]);
      const uint32_t a_k = tc::smem_u32(sAk(k));
      ok = run_phase([&] {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          tc::mma(tm, tc::desc_k(a_k, q), tc::desc_k(sW_a + (KT + k - 1) * kWTile, q), id_fwd, q > 0);
      });
      if (ok) ld64(my_lanes, h);
    }
    if (!ok) {
      timed_out = true;
      break;
    }
    float z = 0.f;
#pragma unroll
    for (int j = 0; j < 64; ++j) z = fmaf(sWout[j], hidden_act(h[j], act), z);
    const float dz = valid ? cur.rec.gsig * act_grad_z(z, out_act) : 0.f;
    // w_out gradient over the warp's samples; G_H = dz * w_out * a'(h_H)
    {
      float v[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) v[j] = dz * hidden_act(h[j], act);
      float s0, s1;
      warp_reduce_scatter64(v, lane, s0, s1, j0_out);
      dwout0 += s0;
      dwout1 += s1;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = hidden_grad(dz * sWout[8 * j + q], h[8 * j + q] > 0.f, act);
      tc::st_chunk_bf16(sG, t, j, v);
    }
    // backward through the hidden layers: G_{k+1} (tile gt) gives
    //   dA_k = G_{k+1} W_k        (A = G K-major, B = W_k MN-major) -> transient columns
    //   dW_k += G_{k+1}^T A_k     (A = G MN-major, M = 128 padded; B = A_k MN-major; K = 128 samples)
    // and G_k = dA_k * a'(a_k) replaces A_k once the dW_k product has completed.
    uint32_t gt = sG_a;
#pragma unroll
    for (int k = H - 1; k >= 1 && ok; --k) {
      const uint32_t a_k = tc::smem_u32(sAk(k));
      const uint32_t wk = sW_a + (KT + k - 1) * kWTile;
      const uint32_t dwk = tm + Plan::T + 64 * (k - 1);
      ok = run_phase([&] {
#pragma unroll
        for (int q = 0; q < 4; ++q) tc::mma(tm, tc::desc_k(gt, q), tc::desc_mn(wk, q, kWTile), id_dA, q > 0);
#pragma unroll
        for (int q = 0; q < 8; ++q)
          tc::mma(dwk, tc::desc_mn(gt, q, pad_lbo), tc::desc_mn(a_k, q, kTile), id_dW, (q > 0) | wacc);
      });
      if (!ok) break;
      ld64(my_lanes, h);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int c = 8 * j + q;
          const uint32_t bit = c < 32 ? (mlo[k] >> c) & 1u : (mhi[k] >> (c - 32)) & 1u;
          v[q] = hidden_grad(h[c], bit != 0, act);
        }
        tc::st_chunk_bf16(sAk(k), t, j, v);
      }
      gt = a_k;
    }
    // dX = G_1 W0 (A = G_1 K-major, B = W0 MN-major over the KT tiles); the
    // layer-0 weight gradient: dW0 += G_1^T X (one X tile), or
    // dW0^T += X^T G_1 (two X tiles as the M = 128 operand, B = G_1 MN-major)
    if (ok)
      ok = run_phase([&] {
#pragma unroll
        for (int q = 0; q < 4; ++q) tc::mma(tm, tc::desc_k(gt, q), tc::desc_mn(sW_a, q, kWTile), id_dX, q > 0);
        if constexpr (KT == 1) {
#pragma unroll
          for (int q = 0; q < 8; ++q)
            tc::mma(dw0, tc::desc_mn(gt, q, pad_lbo), tc::desc_mn(sX_a, q, kTile), id_dW0, (q > 0) | wacc);
        } else {
#pragma unroll
          for (int q = 0; q < 8; ++q)
            tc::mma(dw0, tc::desc_mn(sX_a, q, kTile), tc::desc_mn(gt, q, kTile), id_dW, (q > 0) | wacc);
        }
      });
    if (!ok) {
      timed_out = true;
      break;
    }
    wacc = 1;
    constexpr int NX = (IN + 15) / 16;  // 16-column chunks holding the IN values of dX
    float dx[NX * 16];
#pragma unroll
    for (int c = 0; c < NX; ++c) tc::tmem_ld16(my_lanes + 16 * c, dx + 16 * c);
    tc::tmem_wait_ld();
    if constexpr (kStaged) {
      if (valid) {
        float* dst = stage + ((int64_t)(cur.sched - lo) * a.S + i) * F;
#pragma unroll
        for (int l = 0; l < L; ++l) {
          // evict-first: each staged value is read once, by the scatter pass
          if constexpr (F == 2)
            __stcs(reinterpret_cast<float2*>(dst + l * slots * F), make_float2(dx[2 * l], dx[2 * l + 1]));
          else if constexpr (F == 4)
            __stcs(reinterpret_cast<float4*>(dst + l * slots * F),
                   make_float4(dx[4 * l], dx[4 * l + 1], dx[4 * l + 2], dx[4 * l + 3]));
          else
#pragma unroll
            for (int f = 0; f < F; ++f) dst[l * slots * F + f] = dx[l * F + f];
        }
      }
    } else {
      const uint32_t agg = active ? run_levels(grid, cur.rec.dx, cur.rec.dy, cur.rec.dz, a.run_threshold) : 0u;
      scatter_warp<D, F>(grid, table_grad, p, valid, dx, F, 1, agg, 0, grid.n_levels);
    }
    tc::fence_before();
    __syncthreads();
    if (active) cur.base += 32;
  }
  if (timed_out) {
    if (t == 0) atomicOr(err, 2u);
    tc::mbar_wait(bar, phase);  // let the MMAs in flight retire (bounded) before freeing TMEM
  } else if (wacc) {
    // flush the weight gradients: TMEM lanes 0..63 (warps 0 and 1) hold rows o = 0..63
    tc::fence_after();
    if (warp < 2) {
      const int o = t;
#pragma unroll 1
      for (int k = 1; k < H; ++k) {
        float v[64];
        ld64(my_lanes + Plan::T + 64 * (k - 1), v);
        float* dst = W_grad + 64 * IN + (k - 1) * 64 * 64 + o * 64;
#pragma unroll
        for (int i2 = 0; i2 < 64; ++i2) atomicAdd(dst + i2, v[i2]);
      }
    }
    if constexpr (KT == 1) {
      if (warp < 2) {
        const int o = t;
        float w0[S::INP];
#pragma unroll
        for (int c = 0; c < S::INP / 16; ++c) tc::tmem_ld16(dw0 + ((uint32_t)(32 * warp) << 16) + 16 * c, w0 + 16 * c);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i2 = 0; i2 < IN; ++i2) atomicAdd(W_grad + o * IN + i2, w0[i2]);
      }
    } else if (32 * warp < IN) {  // dW0^T: lane i holds input i's 64 output columns
      float v[64];
      ld64(dw0 + ((uint32_t)(32 * warp) << 16), v);
      if (t < IN) {
#pragma unroll 8
        for (int o = 0; o < 64; ++o) atomicAdd(W_grad + o * IN + t, v[o]);
      }
    }
  }
  {
    float s0, s1;
    float zero[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) zero[j] = 0.f;
    warp_reduce_scatter64(zero, lane, s0, s1, j0_out);  // j0_out of this lane (also when no tile ran)
  }
  red[warp * 64 + j0_out] = dwout0;
  red[warp * 64 + j0_out + 1] = dwout1;
  tc::fence_before();
  __syncthreads();
  if (t < 64)
    atomicAdd(W_grad + 64 * IN + (H - 1) * 64 * 64 + t, red[t] + red[64 + t] + red[128 + t] + red[192 + t]);
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(tm, Plan::kCols);
  }
}

// Lean staged backward for two hidden layers: 128 TMEM columns and 68 KB of
// shared memory per block, so three blocks (12 warps) share an SM.
//   TMEM: [0, 64) the transient result of every phase; [64, 128) the weight
//   gradients, dW1 in lanes 0..63 and dW0 in lanes 64..127.  Both products
//   are M = 128 MMAs whose A operand is a G tile and zeros: dW1 = [G2; 0]^T
//   A1 writes its rows to lanes 0..63 and adds exactly 0 to lanes 64..127,
//   dW0 = [0; G1]^T X the reverse.  The first tile's dW1 product (accumulate
//   off) clears the whole region before dW0 first adds to it.  The zero half
//   of every K step (16 rows of 64 bf16, 2 KB) is one 2 KB zero block, which
//   each step reaches through its own leading-byte offset.
//   Shared memory: W0, W1 | G2 | zero block | A1, then G1 | X.
//   Accumulator rows are read 16 columns at a time; the w_out gradient is a
//   16-column butterfly reduce-scatter per chunk.
template <int D, int F, int ACT>
__global__ void __launch_bounds__(kMixThreads, 3)
bwd_lean_kernel(GridDev grid, const __half* __restrict__ table, const float* __restrict__ W, TrainArgs a,
                const RayRec* __restrict__ recs, const int32_t* __restrict__ slot, unsigned int* __restrict__ ctrl,
                int out_act, float* __restrict__ W_grad, int lo, int hi, float* __restrict__ stage,
                int64_t slots, const int32_t* __restrict__ order, const uint64_t* __restrict__ offs,
                const uint4* __restrict__ xstore, uint32_t xcap) {
  constexpr int IN = 16 * F;
  constexpr int H = 2;
  constexpr int act = ACT;
  static_assert(IN <= 64, "dW0 shares the 64 weight-gradient columns");
  const bool by_pixel = !(ctrl[3] & kFlagDuplicatePixels);
  const unsigned int n_valid = ctrl[6];
  unsigned int* err = ctrl + 2;
  const uint32_t xrows = xstore ? min(xcap, ctrl[7]) : 0u;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = align1024(smem_raw);
  constexpr uint32_t kZero = 2048;    // one K step of a 64-element MN block
  uint8_t* sW = base;                 // W0, W1
  uint8_t* sG = sW + H * kWTile;      // G2
  uint8_t* sZ = sG + kTile;           // zeros (1024-aligned)
  uint8_t* sA = sZ + kZero;           // A1, then G1
  uint8_t* sX = sA + kTile;           // X
  float* sWout = reinterpret_cast<float*>(sX + kTile);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sWout + 64);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  float* red = reinterpret_cast<float*>(tslot + 4);  // [4][64]

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  stage_mixed_weights<16, F, H>(W, sW, sWout);
  {
    uint4* z = reinterpret_cast<uint4*>(sZ);
    for (int e = t; e < (int)(kZero / 16); e += kMixThreads) z[e] = make_uint4(0u, 0u, 0u, 0u);
  }
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
  const uint32_t sG_a = tc::smem_u32(sG), sZ_a = tc::smem_u32(sZ), sA_a = tc::smem_u32(sA), sW_a = tc::smem_u32(sW);
  const uint32_t sX_a = tc::smem_u32(sX);
  constexpr uint32_t id_fwd = tc::idesc_bf16(128, 64, false, false);
  constexpr uint32_t id_dA = tc::idesc_bf16(128, 64, false, true);
  constexpr uint32_t id_dW = tc::idesc_bf16(128, 64, true, true);
  constexpr uint32_t id_dX = tc::idesc_bf16(128, IN, false, true);
  constexpr uint32_t id_dW0 = tc::idesc_bf16(128, IN, true, true);

  uint32_t phase = 0;
  uint32_t wacc = 0;  // the first tile's dW1 product starts the accumulators
  float dwacc[4] = {0.f, 0.f, 0.f, 0.f};  // w_out gradient, column 16c + (lane >> 1) of chunk c
  uint4 xn[IN / 8];                       // the stored row of this thread's sample (prefetched a tile ahead)
  bool pre_ok = false;
  RayCursor cur;
  bool timed_out = false;
  auto run_phase = [&](auto issue) -> bool {
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    if (t == 0) {
      tc::fence_after();
      issue();
      tc::commit(bar);
    }
    const bool to = !tc::mbar_wait(bar, phase);
    phase ^= 1;
    if (__syncthreads_or(to)) return false;
    tc::fence_after();
    return true;
  };
  while (true) {
    const bool active = next_chunk(cur, recs, ctrl + 1, slot, a, by_pixel, lane, lo, hi, order, n_valid, offs, xrows);
    if (!__syncthreads_or(active)) break;
    const int i = cur.base + lane;
    float p[4] = {0.f, 0.f, 0.f, 0.f};
    bool valid = false;
    if (active && i < cur.rec.count) valid = sample_point(cur.rec, i, p);
    if (D == 4) p[3] = a.t;
    if (cur.xrow >= 0) {  // stored rows (warp-uniform branch)
      const uint4* src = xstore + (size_t)(cur.xrow + i) * (IN / 8);
      if (!pre_ok && valid) {
#pragma unroll
        for (int j = 0; j < IN / 8; ++j) xn[j] = __ldcs(src + j);
      }
#pragma unroll
      for (int j = 0; j < IN / 8; ++j) tc::st_chunk_raw(sX, t, j, valid ? xn[j] : make_uint4(0u, 0u, 0u, 0u));
      pre_ok = cur.base + 32 < cur.rec.count;
      if (pre_ok && i + 32 < cur.rec.count) {
#pragma unroll
        for (int j = 0; j < IN / 8; ++j) xn[j] = __ldcs(src + 32 * (IN / 8) + j);
      }
    } else {
      pre_ok = false;
      encode_row<D, F, 16>(grid, table, p, valid, sX, t);
    }
    // layer 0: h1 = X W0^T
    bool ok = run_phase([&] {
#pragma unroll
      for (int q = 0; q < IN / 16; ++q) tc::mma(tm, tc::desc_k(sX_a, q), tc::desc_k(sW_a, q), id_fwd, q > 0);
    });
    if (!ok) {
      timed_out = true;
      break;
    }
    uint32_t m1lo = 0, m1hi = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float h[16];
      tc::tmem_ld16(my_lanes + 16 * c, h);
      tc::tmem_wait_ld();
      float v[8], u[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        v[q] = hidden_act(h[q], act);
        u[q] = hidden_act(h[8 + q], act);
      }
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const uint32_t bit = h[q] > 0.f ? 1u : 0u;
        const int col = 16 * c + q;
        if (col < 32) m1lo |= bit << col; else m1hi |= bit << (col - 32);
      }
      tc::st_chunk_bf16(sA, t, 2 * c, v);
      tc::st_chunk_bf16(sA, t, 2 * c + 1, u);
    }
    // layer 1: h2 = A1 W1^T
    ok = run_phase([&] {
#pragma unroll
      for (int q = 0; q < 4; ++q) tc::mma(tm, tc::desc_k(sA_a, q), tc::desc_k(sW_a + kWTile, q), id_fwd, q > 0);
    });
    if (!ok) {
      timed_out = true;
      break;
    }
    float z = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float h[16];
      tc::tmem_ld16(my_lanes + 16 * c, h);
      tc::tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 16; ++q) z = fmaf(sWout[16 * c + q], hidden_act(h[q], act), z);
    }
    const float dz = valid ? cur.rec.gsig * act_grad_z(z, out_act) : 0.f;
    // second pass over h2: the w_out gradient and G2 = dz * w_out * 1[h2 > 0]
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float h[16];
      tc::tmem_ld16(my_lanes + 16 * c, h);
      tc::tmem_wait_ld();
      float v[16], g[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        v[q] = dz * hidden_act(h[q], act);
        g[q] = hidden_grad(dz * sWout[16 * c + q], h[q] > 0.f, act);
      }
      tc::st_chunk_bf16(sG, t, 2 * c, g);
      tc::st_chunk_bf16(sG, t, 2 * c + 1, g + 8);
      float r8[8], r4[4], r2[2], r1[1];
      detail::rs_step<8>(v, r8, lane, 16);
      detail::rs_step<4>(r8, r4, lane, 8);
      detail::rs_step<2>(r4, r2, lane, 4);
      detail::rs_step<1>(r2, r1, lane, 2);
      dwacc[c] += r1[0] + __shfl_xor_sync(0xffffffffu, r1[0], 1);
    }
    // dA1 = G2 W1 (transient); dW1 += [G2; 0]^T A1 (lanes 0..63 of [64, 128))
    ok = run_phase([&] {
#pragma unroll
      for (int q = 0; q < 4; ++q) tc::mma(tm, tc::desc_k(sG_a, q), tc::desc_mn(sW_a + kWTile, q, kWTile), id_dA, q > 0);
#pragma unroll
      for (int q = 0; q < 8; ++q)  // second M block: the zero block, for every K step
        tc::mma(tm + 64, tc::desc_mn(sG_a, q, sZ_a - (sG_a + 2048u * q)), tc::desc_mn(sA_a, q, kTile), id_dW,
                (q > 0) | wacc);
    });
    if (!ok) {
      timed_out = true;
      break;
    }
    wacc = 1;
    // G1 = dA1 * 1[h1 > 0] replaces A1
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float h[16];
      tc::tmem_ld16(my_lanes + 16 * c, h);
      tc::tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int col = 16 * c + q;
        const uint32_t bit = col < 32 ? (m1lo >> col) & 1u : (m1hi >> (col - 32)) & 1u;
        h[q] = hidden_grad(h[q], bit != 0, act);
      }
      tc::st_chunk_bf16(sA, t, 2 * c, h);
      tc::st_chunk_bf16(sA, t, 2 * c + 1, h + 8);
    }
    // dX = G1 W0 (transient); dW0 += [0; G1]^T X (lanes 64..127 of [64, 64 + IN))
    ok = run_phase([&] {
#pragma unroll
      for (int q = 0; q < 4; ++q) tc::mma(tm, tc::desc_k(sA_a, q), tc::desc_mn(sW_a, q, kWTile), id_dX, q > 0);
#pragma unroll
      for (int q = 0; q < 8; ++q)  // first M block: the zero block; second: K step q of G1
        tc::mma(tm + 64, tc::desc_sw128(sZ_a, sA_a + 2048u * q - sZ_a, 1024u), tc::desc_mn(sX_a, q, kTile), id_dW0,
                1u);
    });
    if (!ok) {
      timed_out = true;
      break;
    }
    {
      float* dst = stage + ((int64_t)(cur.sched - lo) * a.S + i) * F;
#pragma unroll
      for (int c = 0; c < IN / 16; ++c) {
        float dx[16];
        tc::tmem_ld16(my_lanes + 16 * c, dx);  // warp-collective: every lane loads
        tc::tmem_wait_ld();
        if (valid) {
#pragma unroll
          for (int k = 0; k < 16 / F; ++k) {
            const int l = c * (16 / F) + k;  // level
            if constexpr (F == 2)
              __stcs(reinterpret_cast<float2*>(dst + l * slots * F), make_float2(dx[2 * k], dx[2 * k + 1]));
            else
              __stcs(reinterpret_cast<float4*>(dst + l * slots * F),
                     make_float4(dx[4 * k], dx[4 * k + 1], dx[4 * k + 2], dx[4 * k + 3]));
          }
        }
      }
    }
    tc::fence_before();
    __syncthreads();
    if (active) cur.base += 32;
  }
  if (timed_out) {
    if (t == 0) atomicOr(err, 2u);
    tc::mbar_wait(bar, phase);  // let the MMAs in flight retire (bounded) before freeing TMEM
  } else if (wacc) {
    tc::fence_after();
    if (warp < 2) {  // dW1 rows o = t in lanes 0..63
      float v[64];
      ld64(my_lanes + 64, v);
      float* dst = W_grad + 64 * IN + t * 64;
#pragma unroll
      for (int j = 0; j < 64; ++j) atomicAdd(dst + j, v[j]);
    } else {  // dW0 rows o = t - 64 in lanes 64..127
      float v[IN];
#pragma unroll
      for (int c = 0; c < IN / 16; ++c) tc::tmem_ld16(my_lanes + 64 + 16 * c, v + 16 * c);
      tc::tmem_wait_ld();
      float* dst = W_grad + (t - 64) * IN;
#pragma unroll
      for (int j = 0; j < IN; ++j) atomicAdd(dst + j, v[j]);
    }
  }
  if (!(lane & 1)) {
#pragma unroll
    for (int c = 0; c < 4; ++c) red[warp * 64 + 16 * c + (lane >> 1)] = dwacc[c];
  }
  tc::fence_before();
  __syncthreads();
  if (t < 64) atomicAdd(W_grad + 64 * IN + 64 * 64 + t, red[t] + red[64 + t] + red[128 + t] + red[192 + t]);
  if (warp == 0) {
    tc::fence_after();
    tc::tmem_dealloc(tm, 128);
  }
}

// Applies staged encoding gradients of the rays with scheduling index in
// [lo, hi) to the fp32 gradient table, levels [l0, l1) only: a pass touches a
// slice of the gradient table small enough to stay in L2.  Warp per 32
// consecutive samples of a ray (the backward's order, so runs of equal cells
// are merged the same way); no shared memory or TMEM, so many warps per SM
// keep many reductions in flight.
template <int D, int F>
__global__ void __launch_bounds__(kScatterThreads)
scatter_stage_kernel(GridDev grid, TrainArgs a, const RayRec* __restrict__ recs, const int32_t* __restrict__ slot,
                     unsigned int* __restrict__ ctrl, const float* __restrict__ stage, int64_t slots, int lo, int hi,
                     int l0, int l1, float* __restrict__ table_grad, const int32_t* __restrict__ order) {
  const bool by_pixel = !(ctrl[3] & kFlagDuplicatePixels);
  const unsigned int n_valid = ctrl[6];
  const int lane = threadIdx.x & 31;
  RayCursor cur;
  while (next_chunk(cur, recs, ctrl + 5, slot, a, by_pixel, lane, lo, hi, order, n_valid)) {
    const int i = cur.base + lane;
    float p[4] = {0.f, 0.f, 0.f, 0.f};
    bool valid = false;
    if (i < cur.rec.count) valid = sample_point(cur.rec, i, p);
    if (D == 4) p[3] = a.t;
    const float* dsrc = stage + ((int64_t)(cur.sched - lo) * a.S + i) * F;
    scatter_warp<D, F, true>(grid, table_grad, p, valid, dsrc, slots * F, 1,
                             run_levels(grid, cur.rec.dx, cur.rec.dy, cur.rec.dz, a.run_threshold), l0, l1);
    cur.base += 32;
  }
}

// Builds the fp16 time slice of every level (grid y = level): slice entry k
// blends the entries of the two time vertices; dense levels' padding is zero.
template <int F>
__global__ void time_slice_kernel(TimeSlice s, const __half* __restrict__ t4, __half* __restrict__ t3) {
  const int l = blockIdx.y;
  const bool hashed = (s.g3.hashed_bits >> l) & 1u;
  const int64_t n = (l + 1 < s.g3.n_levels ? s.g3.offset[l + 1] : s.g3.total_entries) - s.g3.offset[l];
  const float w0 = s.w0[l], w1 = s.w1[l];
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    __half* dst = t3 + (s.g3.offset[l] + k) * F;
    if (k >= s.n_real[l]) {
#pragma unroll
      for (int f = 0; f < F; ++f) dst[f] = __float2half_rn(0.f);
      continue;
    }
    const int64_t e0 = hashed ? (int64_t)((uint64_t)k ^ (uint64_t)s.c0[l]) : k + s.c0[l];
    const int64_t e1 = hashed ? (int64_t)((uint64_t)k ^ (uint64_t)s.c1[l]) : k + s.c1[l];
    const __half* a = t4 + (s.off4[l] + e0) * F;
    const __half* b = t4 + (s.off4[l] + e1) * F;
#pragma unroll
    for (int f = 0; f < F; ++f) dst[f] = __float2half_rn(fmaf(w0, __half2float(a[f]), w1 * __half2float(b[f])));
  }
}

// Adds the slice-shaped gradient g3 to the 4D gradient table at the two time
// vertices (grid y = level).  Hashed levels: one thread per 4D entry gathers
// its two slice entries (an XOR is its own inverse, so no two threads write
// the same entry); dense levels: one thread per slice entry writes its two
// vertices, which lie in different t slabs.
template <int F>
__global__ void time_spread_kernel(TimeSlice s, const float* __restrict__ g3, float* __restrict__ g4) {
  const int l = blockIdx.y;
  const bool hashed = (s.g3.hashed_bits >> l) & 1u;
  const int64_t n = s.n_real[l];
  const float w0 = s.w0[l], w1 = s.w1[l];
  const float* src = g3 + s.g3.offset[l] * F;
  float* dst = g4 + s.off4[l] * F;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    if (hashed) {
      const float* a = src + (int64_t)((uint64_t)k ^ (uint64_t)s.c0[l]) * F;
      const float* b = src + (int64_t)((uint64_t)k ^ (uint64_t)s.c1[l]) * F;
#pragma unroll
      for (int f = 0; f < F; ++f) dst[k * F + f] += fmaf(w0, a[f], w1 * b[f]);
    } else {
#pragma unroll
      for (int f = 0; f < F; ++f) {
        const float v = src[k * F + f];
        dst[(k + s.c0[l]) * F + f] += w0 * v;
        dst[(k + s.c1[l]) * F + f] += w1 * v;
      }
    }
  }
}


// Level groups of the staged scatter: consecutive levels whose fp32 gradient
// slices add up to at most the tuning's scatter_group_bytes (48 MiB by default).
template <int D, int F, int L, int H, int ACT>
int run_mixed(const NectbGeometry& geo, const GridDev& grid, const __half* table, const float* W,
              const TrainArgs& args, Workspace ws, int out_act, float* table_grad, float* W_grad, float* y_pred,
              float* loss, cudaStream_t s) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const NectbTuning tune = current_tuning();
  if constexpr (D == 4) {
    // Training with staging: the 3D kernels on the time slice at the batch's t
    // (queries and steps without staging room keep the 4D kernels).  The slice
    // and its gradient sit at the end of the staging region.  A re-projection
    // piece (forward only, fwd_warpgroups > 0) builds only the fp16 slice, at
    // the start of its staging region, and runs without staging.
    const bool piece = args.fwd_warpgroups > 0 && !table_grad;
    const size_t sb = piece ? slice_half_bytes(grid) : slice_bytes(grid);
    const size_t need = piece ? sb + 512 : sb + order_bytes(args.num_rays, args.n_pixels) + (size_t(1) << 20);
    if (tune.time_slice && args.max_blocks == 0 && ws.stage && ws.stage_bytes >= need) {
      const TimeSlice ts = make_time_slice(grid, args.t);
      const int64_t n3 = ts.g3.total_entries;
      Workspace ws3 = ws;
      __half* t3;
      if (piece) {  // on a 512-byte boundary (a texture's alignment)
        t3 = reinterpret_cast<__half*>((reinterpret_cast<uintptr_t>(ws.stage) + 511) & ~uintptr_t(511));
        ws3.stage = nullptr;
        ws3.stage_bytes = 0;
      } else {
        // the slice starts on a 512-byte boundary (a texture's alignment)
        const uintptr_t st = reinterpret_cast<uintptr_t>(ws.stage);
        ws3.stage_bytes = (size_t)(((st + ws.stage_bytes - sb) & ~uintptr_t(511)) - st);
        t3 = reinterpret_cast<__half*>(reinterpret_cast<char*>(ws.stage) + ws3.stage_bytes);
      }
      float* g3 =
          piece ? nullptr : reinterpret_cast<float*>(reinterpret_cast<char*>(t3) + align256((size_t)n3 * F * 2));
      int64_t max_level = 0;
      for (int l = 0; l < grid.n_levels; ++l) max_level = std::max(max_level, ts.n_real[l] + 8);
      const dim3 sgrid((unsigned)std::min<int64_t>(ceil_div(max_level, 256), 1024), (unsigned)grid.n_levels);
      if (args.phase & kPhaseForward) {
        {
          ProfScope ps(kProfSlice, s);
          time_slice_kernel<F><<<sgrid, 256, 0, s>>>(ts, table, t3);
        }
        if (int rc = launch_status("time_slice_kernel")) return rc;
      }
      const bool bwd = table_grad && (args.phase & kPhaseBackward);
      if (bwd)
        if (int rc = cuda_status(cudaMemsetAsync(g3, 0, (size_t)n3 * F * sizeof(float), s), "memset slice gradient"))
          return rc;
      if (int rc = run_mixed<3, F, L, H, ACT>(geo, ts.g3, t3, W, args, ws3, out_act, bwd ? g3 : nullptr, W_grad,
                                              y_pred, loss, s))
        return rc;
      if (bwd) {
        {
          ProfScope ps(kProfSlice, s);
          time_spread_kernel<F><<<sgrid, 256, 0, s>>>(ts, g3, table_grad);
        }
        if (int rc = launch_status("time_spread_kernel")) return rc;
      }
      return NECTB_OK;
    }
  }
  (void)geo;
  TrainArgs a = args;
  a.run_threshold = D == 4 ? tune.run_threshold_4d : tune.run_threshold_3d;
  const size_t group_bytes = (size_t)tune.scatter_group_bytes;
  // forward: one block of `wgs` warpgroups per SM when training; queries
  // (which share SMs with serving kernels) one warpgroup per block, or the
  // caller's warpgroups per SM
  const bool shares_sms = a.max_blocks > 0 || a.fwd_warpgroups > 0;
  constexpr int kMaxWg = FwdShape<D, L, F, H>::kMaxWarpgroups;
  const int wgs = a.max_blocks > 0       ? 1
                  : a.fwd_warpgroups > 0 ? std::min(a.fwd_warpgroups, kMaxWg)
                                         : std::min(tune.forward_blocks_per_sm, kMaxWg);
  int fblocks = a.max_blocks > 0 ? std::max(1, std::min<int>(std::min(tune.forward_blocks_per_sm, kMaxWg) * sms,
                                                             (int)ceil_div(a.num_rays, 4)))
                                 : std::max(1, std::min<int>(sms, (int)ceil_div(a.num_rays, 4 * wgs)));
  // the general backward: two blocks per SM of 256 TMEM columns, one of 512
  const int bwd_per_sm = BwdPlan<L, F, H>::kCols == 512u ? 1 : std::min(tune.backward_blocks_per_sm, 2);
  int blocks = std::max(1, std::min<int>(bwd_per_sm * sms, (int)ceil_div(a.num_rays, 4)));
  if (a.max_blocks > 0) {
    fblocks = std::min(fblocks, a.max_blocks);
    blocks = std::min(blocks, a.max_blocks);
  }
  using Shape = InShape<L, F>;
  constexpr int IN = Shape::IN, KT = Shape::KT;
  GridDev gt = grid;  // the grid with a texture over the fp16 table for the encoders' gathers
  if (a.texture)
    gt.tex = table_texture(table, (size_t)grid.total_entries * F * sizeof(__half), F * (int)sizeof(__half));
  const int R = a.num_rays;
  // staging region: ray order and sample offsets, the encoding store (bf16
  // input rows with their zero padding), then dL/d(encoding) of one round of
  // per_round rays
  const StageLayout SL = stage_layout(ws, R, a.n_pixels, a.S, Shape::INP * sizeof(__nv_bfloat16),
                                      (size_t)a.S * IN * sizeof(float), tune.staged_rounds,
                                      tune.encoding_store != 0 && !shares_sms);
  auto run_order = [&]() -> int {
    ProfScope ps(kProfOrder, s);
    const int n_blocks = order_blocks(R, a.n_pixels);
    order_count_kernel<<<n_blocks, kOrderBlock, 0, s>>>(ws.slot, ws.rays, ws.counters, R, a.n_pixels, SL.block_sums,
                                                        SL.block_samples);
    order_scan_kernel<<<1, kOrderBlock, 0, s>>>(SL.block_sums, SL.block_samples, n_blocks, ws.counters);
    order_compact_kernel<<<n_blocks, kOrderBlock, 0, s>>>(ws.slot, ws.rays, ws.counters, R, a.n_pixels, SL.block_sums,
                                                          SL.block_samples, SL.order, SL.offs);
    return launch_status("order kernels");
  };
  if (a.phase & kPhaseForward) {
    // with an encoding store the forward runs the rays in rank order and keeps their rows
    if (SL.xstore)
      if (int rc = run_order()) return rc;
    auto k = fwd_mixed_kernel<D, F, L, H, ACT>;
    const size_t smem = 1024 + (KT + H - 1) * kWTile + wgs * KT * kTile + 64 * 4 + kFwdBlocksPerSM * 8 + 16 +
                        4 * kFwdBlocksPerSM * 4;
    set_smem(k, smem, shares_sms);
    {
      ProfScope ps(kProfForward, s);
      k<<<fblocks, kMixThreads * wgs, smem, s>>>(gt, table, W, a, ws.rays, ws.slot, ws.counters, out_act, y_pred, loss,
                                           SL.xstore ? SL.order : nullptr, SL.offs, SL.xstore, SL.xcap);
    }
    if (int rc = launch_status("fwd_mixed_kernel")) return rc;
  }
  if (!table_grad || !(a.phase & kPhaseBackward)) return NECTB_OK;  // forward only (queries, split step)
  // at least 80 KB keeps at most two blocks (2 x 256 TMEM columns) per SM;
  // the 512-column plans take more than half of the shared memory
  const size_t bsmem = std::max<size_t>(BwdPlan<L, F, H>::smem, 80 * 1024);
  if (SL.per_round <= 0) {
    // fused single pass: the backward scatters its own gradients
    auto k = bwd_mixed_kernel<D, F, L, H, false, ACT>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsmem);
    ProfScope ps(kProfBackward, s);
    k<<<blocks, kMixThreads, bsmem, s>>>(gt, table, W, a, ws.rays, ws.slot, ws.counters, out_act, table_grad,
                                         W_grad, 0, 0x7fffffff, nullptr, 0, nullptr, nullptr, nullptr, 0u);
    return launch_status("bwd_mixed_kernel");
  }
  // the order is a function of the prepared rays alone: computed again unless
  // this call's forward just did
  if (!((a.phase & kPhaseForward) && SL.xstore))
    if (int rc = run_order()) return rc;
  const int64_t per_round = SL.per_round;
  float* stage = SL.stage;
  const int32_t* order = SL.order;
  // two passes per round of Q ordered rays: the tensor-core backward stages
  // dL/d(encoding), then one scatter pass per level group
  int group_start[NECTB_MAX_LEVELS + 1], n_groups = 0;
  {
    size_t acc = 0;
    for (int l = 0; l < grid.n_levels; ++l) {
      const int64_t next = l + 1 < grid.n_levels ? grid.offset[l + 1] : grid.total_entries;
      const size_t bytes = (size_t)(next - grid.offset[l]) * F * sizeof(float);
      if (l == 0 || acc + bytes > group_bytes) {
        group_start[n_groups++] = l;
        acc = 0;
      }
      acc += bytes;
    }
    group_start[n_groups] = grid.n_levels;
  }
  // tensor-core pass of a round: the lean kernel for two hidden layers over at
  // most 64 inputs (up to three blocks per SM), else the general one (two)
  constexpr bool kLean = H == 2 && L == 16 && IN <= 64;
  const size_t lsmem = 1024 + 2 * kWTile + 3 * kTile + 2048 + 64 * 4 + 64 + 4 * 64 * 4;
  const int lblocks = std::max(1, std::min<int>(tune.backward_blocks_per_sm * sms, (int)ceil_div(a.num_rays, 4)));
  if constexpr (kLean)
    set_smem(bwd_lean_kernel<D, F, ACT>, lsmem, false);
  else
    cudaFuncSetAttribute(bwd_mixed_kernel<D, F, L, H, true, ACT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)bsmem);
  auto ks = scatter_stage_kernel<D, F>;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ks, kScatterThreads, 0);
  if (tune.scatter_blocks_per_sm > 0) per_sm = std::min(per_sm, tune.scatter_blocks_per_sm);
  const int sblocks = sms * std::max(per_sm, 1);
  const int64_t slots = per_round * a.S;
  for (int64_t lo = 0; lo < R; lo += per_round) {
    const int hi = (int)std::min<int64_t>(R, lo + per_round);
    if (int rc = cuda_status(cudaMemsetAsync(ws.counters + 1, 0, sizeof(unsigned int), s), "memset cursor")) return rc;
    {
      ProfScope ps(kProfBackward, s);
      if constexpr (kLean)
        bwd_lean_kernel<D, F, ACT><<<lblocks, kMixThreads, lsmem, s>>>(gt, table, W, a, ws.rays, ws.slot,
                                                                       ws.counters, out_act, W_grad, (int)lo, hi,
                                                                       stage, slots, order, SL.offs, SL.xstore,
                                                                       SL.xcap);
      else
        bwd_mixed_kernel<D, F, L, H, true, ACT><<<blocks, kMixThreads, bsmem, s>>>(
            gt, table, W, a, ws.rays, ws.slot, ws.counters, out_act, table_grad, W_grad, (int)lo, hi, stage, slots,
            order, SL.offs, SL.xstore, SL.xcap);
    }
    if (int rc = launch_status("bwd_mixed_kernel")) return rc;
    for (int gi = 0; gi < n_groups; ++gi) {
      if (int rc = cuda_status(cudaMemsetAsync(ws.counters + 5, 0, sizeof(unsigned int), s), "memset cursor"))
        return rc;
      {
        ProfScope ps(kProfScatter, s);
        ks<<<sblocks, kScatterThreads, 0, s>>>(grid, a, ws.rays, ws.slot, ws.counters, stage, slots, (int)lo, hi,
                                               group_start[gi], group_start[gi + 1], table_grad, order);
      }
      if (int rc = launch_status("scatter_stage_kernel")) return rc;
    }
  }
  return NECTB_OK;
}

}  // namespace

int train_mixed(const NectbGeometry& geo, const GridDev& grid, const NectbMLP& mlp, const void* table,
                const float* W, int nW, const TrainArgs& a, Workspace ws, float* table_grad, float* W_grad,
                float* y_pred, float* loss, cudaStream_t s) {
  (void)nW;
  const int D = grid.n_dims, F = grid.n_features, L = grid.n_levels;
  const int H = mlp.n_hidden_layers;
  if (H < 2)
    return set_error(NECTB_ERR_INVALID, "mixed path: needs at least 2 hidden layers (got %d)", H);
  const __half* tab = (const __half*)table;
  const int act = mlp.activation, oact = mlp.output_activation;
  // the hidden activation is a template constant of the kernels: ReLU for
  // every shape, LeakyReLU for the reference's default static model too
  const int rc = dispatch_shape(D, F, L, H, [&](auto d, auto f, auto l, auto h) {
    if (act == NECTB_ACT_RELU)
      return run_mixed<d(), f(), l(), h(), NECTB_ACT_RELU>(geo, grid, tab, W, a, ws, oact, table_grad, W_grad,
                                                            y_pred, loss, s);
    if constexpr (l() != 16) {
      if (act == NECTB_ACT_LEAKY_RELU)
        return run_mixed<d(), f(), l(), h(), NECTB_ACT_LEAKY_RELU>(geo, grid, tab, W, a, ws, oact, table_grad,
                                                                    W_grad, y_pred, loss, s);
    }
    return set_error(NECTB_ERR_INVALID, "mixed path: hidden activation %d is not instantiated for this shape (ReLU "
                     "for every shape, LeakyReLU for 19 levels x 4 features)", act);
  });
  if (rc != kUnsupportedShape) return rc;
  return set_error(NECTB_ERR_INVALID, "mixed path: unsupported model shape (n_dims %d, n_features %d, n_levels %d, "
                   "hidden %d)", D, F, L, H);
}

// A texture object over an fp16 table of entry_bytes-byte entries (4: two
// features, 8: four; created once per buffer and kept), or 0 when the table
// exceeds the 1D linear texture width or is not aligned for a texture.
cudaTextureObject_t table_texture(const void* ptr, size_t bytes, int entry_bytes) {
  static std::mutex mu;
  static std::vector<std::tuple<const void*, size_t, cudaTextureObject_t, int>> cache;
  std::lock_guard<std::mutex> lk(mu);
  for (auto& e : cache)
    if (std::get<0>(e) == ptr && std::get<1>(e) == bytes && std::get<3>(e) == entry_bytes) return std::get<2>(e);
  int dev = 0, maxw = 0, align = 512;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxTexture1DLinearWidth, dev);
  cudaDeviceGetAttribute(&align, cudaDevAttrTextureAlignment, dev);
  if (bytes / entry_bytes > (size_t)maxw || align <= 0 || (reinterpret_cast<uintptr_t>(ptr) % (uintptr_t)align) != 0)
    return 0;
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeLinear;
  rd.res.linear.devPtr = const_cast<void*>(ptr);
  rd.res.linear.desc = entry_bytes == 8 ? cudaCreateChannelDesc<uint2>() : cudaCreateChannelDesc<unsigned int>();
  rd.res.linear.sizeInBytes = bytes;
  cudaTextureDesc td = {};
  td.readMode = cudaReadModeElementType;
  cudaTextureObject_t tex = 0;
  if (cudaCreateTextureObject(&tex, &rd, &td, nullptr) != cudaSuccess) {
    cudaGetLastError();  // no texture: the loads take the LSU path
    return 0;
  }
  cache.emplace_back(ptr, bytes, tex, entry_bytes);
  return tex;
}

// The fp16 time slice of a 4D fp16 table at t (layout make_time_slice(grid, t).g3).
int launch_time_slice(const GridDev& grid, const __half* table, float t, __half* slice, cudaStream_t s) {
  const TimeSlice ts = make_time_slice(grid, t);
  int64_t max_level = 0;
  for (int l = 0; l < grid.n_levels; ++l) max_level = std::max(max_level, ts.n_real[l] + 8);
  const dim3 sgrid((unsigned)std::min<int64_t>(ceil_div(max_level, 256), 1024), (unsigned)grid.n_levels);
  ProfScope ps(kProfSlice, s);
  if (grid.n_features == 2)
    time_slice_kernel<2><<<sgrid, 256, 0, s>>>(ts, table, slice);
  else if (grid.n_features == 4)
    time_slice_kernel<4><<<sgrid, 256, 0, s>>>(ts, table, slice);
  else
    return set_error(NECTB_ERR_INVALID, "time slice: %d features per level (2 or 4)", grid.n_features);
  return launch_status("time_slice_kernel");
}

}  // namespace nectb
