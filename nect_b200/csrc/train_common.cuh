// Pieces shared by the plain (fp32 SIMT) and mixed (bf16 tcgen05) fused
// training kernels: per-ray records, the ray-preparation kernel, the ray
// scheduler, sample regeneration and the workspace layout.
#pragma once
#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "geometry.cuh"
#include "hashgrid.cuh"

namespace nectb {

// Everything a fused kernel needs to regenerate the samples of one ray
// without touching positions in memory.  64 bytes.
struct RayRec {
  double sx, sy, sz;   // first sample (normalised, clamped), fp64 as in the reference
  double dx, dy, dz;   // spacing
  int32_t count;       // samples written by the reference loop
  float scale;         // distances[r] / max_distance_traveled (base_trainer.py:552-554)
  float y;             // measured value proj[perm[start + r]]
  float gsig;          // dL/dsigma for every sample of the ray (set by the forward)
};
static_assert(sizeof(RayRec) == 64, "RayRec must be 64 bytes");

enum { kPhaseForward = 1, kPhaseBackward = 2 };

struct TrainArgs {
  const int64_t* perm;
  int64_t perm_len;
  int64_t start;
  int num_rays;
  int n_pixels;  // nDetector[0] * nDetector[1]
  int S;
  float angle;
  float t;
  float maxd;
  int uniform;
  float max_dist;
  const float* jitter;
  const float* det_off;
  const float* projection;
  int loss_type;
  float loss_scale;
  int max_blocks;  // > 0: cap on the persistent grids (queries); 0: default
  int phase = kPhaseForward | kPhaseBackward;  // which half of the step to run
  float run_threshold = 0.75f;                 // run merging of the scatter (set from the tuning)
};

enum : unsigned int { kFlagDuplicatePixels = 1u };

// The two-pass mixed backward: the most rounds a staging buffer may need
// before the fused single-pass backward is used instead (the recommended
// staging is sized for NectbTuning::staged_rounds, 4 by default).
constexpr int kMaxStagedRounds = 64;
constexpr size_t kStagingCap = size_t(16) << 30;  // largest staging buffer recommended
constexpr int kOrderBlock = 1024;                  // threads of the ray-order kernels

// Bytes at the front of the staging region for the ray order and its block sums.
inline size_t order_bytes(int R, int P) {
  const size_t n_blocks = (size_t)(std::max(R, P) + kOrderBlock - 1) / kOrderBlock;
  return (((size_t)R * 4 + 255) & ~size_t(255)) + (((n_blocks + 1) * 4 + 255) & ~size_t(255));
}

// Workspace: RayRec[R] | slot[P] (int32: batch index of the ray through each
// detector pixel, -1 if none) | 64-byte control block (scheduling cursors of
// the forward and backward, error word, flags).
// Any workspace bytes beyond workspace_bytes() (from a 256-byte boundary) are
// the staging buffer of the two-pass mixed backward.
struct Workspace {
  RayRec* rays;
  int32_t* slot;
  unsigned int* counters;  // [0] forward cursor, [1] backward cursor, [2] error word, [3] flags,
                           // [5] scatter cursor
  float* stage = nullptr;
  size_t stage_bytes = 0;
};

inline size_t workspace_bytes(int R, int P) { return (size_t)R * sizeof(RayRec) + (size_t)P * 4 + 256; }

inline Workspace carve_workspace(void* ws, int R, int P, size_t size = 0) {
  Workspace w;
  w.rays = (RayRec*)ws;
  w.slot = (int32_t*)((char*)ws + (size_t)R * sizeof(RayRec));
  w.counters = (unsigned int*)((char*)w.slot + (((size_t)P * 4 + 63) & ~size_t(63)));
  const size_t base = (workspace_bytes(R, P) + 255) & ~size_t(255);
  if (size > base) {
    w.stage = (float*)((char*)ws + base);
    w.stage_bytes = size - base;
  }
  return w;
}

// Warp per ray: set-up, sample count (warp ballot), measured value, scale;
// claims the ray's detector pixel in slot[]; finalises rays without samples
// (y_pred = 0, their loss term and gradient).
__global__ void ray_prep_kernel(NectbGeometry g, TrainArgs a, RayRec* __restrict__ recs, int32_t* __restrict__ slot,
                                unsigned int* __restrict__ ctrl, float* __restrict__ y_pred, float* __restrict__ loss);

// Position of sample i of a prepared ray, after the Projector clamp
// (projector.py:127); returns false for the zero points the trainer drops
// (base_trainer.py:523).
__device__ __forceinline__ bool sample_point(const RayRec& r, int i, float* p) {
  const float px = r.sx + i * r.dx;
  const float py = r.sy + i * r.dy;
  const float pz = r.sz + i * r.dz;
  p[0] = clamp01f(pz);
  p[1] = clamp01f(py);
  p[2] = clamp01f(px);
  return !(p[0] == 0.f && p[1] == 0.f && p[2] == 0.f);
}

__device__ __forceinline__ RayRec load_ray(const RayRec* recs, int r) { return recs[r]; }

// Warp-uniform scheduler: hands out the rays of the batch that have samples,
// in detector-pixel order (neighbouring rays run together, so the blocks in
// flight touch a compact part of the tables and the L2 keeps it), or in batch
// order when the batch repeats a pixel.  Returns -1 when none are left.
// The scheduling index (pixel, or batch position) of the returned ray is
// written to *sched; only indices in [lo, hi) are handed out (a round of the
// staged backward), the cursor counting from lo.
__device__ __forceinline__ int next_ray(unsigned int* cursor, const int32_t* __restrict__ slot,
                                        const RayRec* __restrict__ recs, int R, int P, bool by_pixel, int lane,
                                        int lo = 0, int hi = 0x7fffffff, int* sched = nullptr) {
  const unsigned int end = (unsigned)min(hi, by_pixel ? P : R);
  while (true) {
    unsigned int idx = 0;
    if (lane == 0) idx = (unsigned)lo + atomicAdd(cursor, 1u);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= end) return -1;
    if (sched) *sched = (int)idx;
    if (by_pixel) {
      const int r = slot[idx];
      if (r >= 0) return r;
    } else {
      if (recs[idx].count > 0) return (int)idx;
    }
  }
}

// The rays with samples in scheduling order, for the two-pass backward's
// rounds of equal ray counts: order[rank] = ray, ranks 0..ctrl[6]-1.  Three
// launches over the scheduling indices (pixels, or batch positions when the
// batch repeats a pixel): per-block counts, one block scanning them, and the
// per-block compaction, so pixel order is kept.
__global__ void order_count_kernel(const int32_t* __restrict__ slot, const RayRec* __restrict__ recs,
                                   const unsigned int* __restrict__ ctrl, int R, int P,
                                   unsigned int* __restrict__ block_sums);
__global__ void order_scan_kernel(unsigned int* __restrict__ block_sums, int n_blocks, unsigned int* __restrict__ ctrl);
__global__ void order_compact_kernel(const int32_t* __restrict__ slot, const RayRec* __restrict__ recs,
                                     const unsigned int* __restrict__ ctrl, int R, int P,
                                     const unsigned int* __restrict__ block_sums, int32_t* __restrict__ order);

// Scheduler over ranks [lo, hi) of the ordered rays (one round); the rank of
// the returned ray is written to *sched.  Returns -1 when none are left.
__device__ __forceinline__ int next_ray_ranked(unsigned int* cursor, const int32_t* __restrict__ order,
                                               unsigned int n_valid, int lo, int hi, int lane, int* sched) {
  unsigned int idx = 0;
  if (lane == 0) idx = (unsigned)lo + atomicAdd(cursor, 1u);
  idx = __shfl_sync(0xffffffffu, idx, 0);
  if (idx >= min((unsigned)hi, n_valid)) return -1;
  *sched = (int)idx;
  return order[idx];
}

// Loss gradient dL/dy_pred for one ray (mean over rays, nect/config.py:481-497),
// times the ray's scale (dy_pred/dsigma).
__device__ __forceinline__ float loss_grad(float y_pred, float y, int loss_type, int R, float scale) {
  const float d = y_pred - y;
  float g;
  if (loss_type == 1)
    g = (d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f)) / (float)R;
  else
    g = 2.f * d / (float)R;
  return g * scale;
}

__device__ __forceinline__ float loss_term(float y_pred, float y, int loss_type) {
  const float d = y_pred - y;
  return loss_type == 1 ? fabsf(d) : d * d;
}

}  // namespace nectb
