// Pieces shared by the plain (fp32 SIMT) and mixed (bf16 tcgen05) fused
// training kernels: per-ray records, the ray-preparation kernel, the ray
// scheduler, sample regeneration and the workspace layout.
#pragma once
#include <algorithm>
#include <cmath>
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

// Continuous-scan steps: at most this many sub-angles per batch.
constexpr int kMaxSubAngles = 32;

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
  // > 0: the forward runs one block of this many warpgroups per SM under the
  // shared-SM carveout (re-projection pieces beside serving kernels); 0: the tuning's
  int fwd_warpgroups = 0;
  // the encoders may fetch corners through a texture object over the table
  // (false: loads only, no texture object created)
  bool texture = true;
  int phase = kPhaseForward | kPhaseBackward;  // which half of the step to run
  float run_threshold = 0.75f;                 // run merging of the scatter (set from the tuning)
  // Continuous scan (sub > 1): num_rays = sub * (pixels of the batch) virtual
  // rays, sub-angle-major (ray v = j * pixels + r is pixel r at sub_angle[j],
  // with jitter[v] and det_off[2v..2v+1]); n_pixels = sub * detector pixels,
  // slot index = pixel * sub + j.
  int sub = 1;
  float sub_angle[kMaxSubAngles];
};

enum : unsigned int { kFlagDuplicatePixels = 1u };

// The two-pass mixed backward: the most rounds a staging buffer may need
// before the fused single-pass backward is used instead (the recommended
// staging is sized for NectbTuning::staged_rounds, 4 by default).
constexpr int kMaxStagedRounds = 64;
constexpr size_t kStagingCap = size_t(16) << 30;  // largest staging buffer recommended
constexpr int kOrderBlock = 1024;                  // threads of the ray-order kernels

// Stored encodings: the forward writes each sample's bf16 MLP input row, which
// the backward reads back instead of gathering the tables again.  Largest
// store the recommended staging size includes.
constexpr size_t kEncodingStoreCap = size_t(80) << 30;

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
inline int order_blocks(int R, int P) { return (std::max(R, P) + kOrderBlock - 1) / kOrderBlock; }

// Bytes at the front of the staging region: the ray order, its block sums,
// the sample offset of every ranked ray and their block sums.
inline size_t order_bytes(int R, int P) {
  const size_t nb = (size_t)order_blocks(R, P) + 1;
  return align256((size_t)R * 4) + align256(nb * 4) + align256((size_t)R * 8) + align256(nb * 8);
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
                           // [5] scatter cursor, [6] rays with samples, [7] encoding-store rows
                           // the forward filled, [8] forward loss sum (split step)
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

// Split of the staging region of the two-pass mixed backward:
//   order[R] int32 | block sums | offs[R] uint64 (first stored row of each
//   ranked ray) | block sums | encoding store [xcap rows of row_bytes] |
//   staged dL/d(encoding) of one round of per_round rays (per_ray bytes each).
// The staged rounds take the recommended size for `rounds` rounds (capped at
// kStagingCap) and the encoding store the rest, up to R * S rows; when that
// leaves less than one ray's rows there is no store and the rounds take the
// whole region.  per_round == 0: no staging (the fused single-pass backward).
// The store starts at the same address whatever the split, so a backward half
// reading rows [0, min(its xcap, the forward's)) never reads its own staging.
struct StageLayout {
  int32_t* order = nullptr;
  unsigned int* block_sums = nullptr;
  uint64_t* offs = nullptr;
  unsigned long long* block_samples = nullptr;
  uint4* xstore = nullptr;
  uint32_t xcap = 0;  // rows of the encoding store
  float* stage = nullptr;
  int64_t per_round = 0;
};

inline size_t staged_round_bytes(int R, int rounds, size_t per_ray) {
  const int64_t per_round = (R + rounds - 1) / rounds;
  return std::min((size_t)per_round * per_ray, kStagingCap / per_ray * per_ray);
}

// store == false: no encoding store whatever the buffer size (the backward
// recomputes every sample's encoding from the tables).
inline StageLayout stage_layout(const Workspace& ws, int R, int P, int S, size_t row_bytes, size_t per_ray,
                                int rounds, bool store = true) {
  StageLayout L;
  const size_t ob = order_bytes(R, P);
  if (!ws.stage || ws.stage_bytes <= ob || R <= 0) return L;
  char* p = reinterpret_cast<char*>(ws.stage);
  const size_t nb = (size_t)order_blocks(R, P) + 1;
  L.order = reinterpret_cast<int32_t*>(p);
  L.block_sums = reinterpret_cast<unsigned int*>(p + align256((size_t)R * 4));
  L.offs = reinterpret_cast<uint64_t*>(p + align256((size_t)R * 4) + align256(nb * 4));
  L.block_samples = reinterpret_cast<unsigned long long*>(p + align256((size_t)R * 4) + align256(nb * 4) +
                                                          align256((size_t)R * 8));
  const size_t avail = ws.stage_bytes - ob;
  const size_t want = staged_round_bytes(R, rounds, per_ray);
  size_t xbytes = 0;
  if (store && avail >= want + (size_t)S * row_bytes + 256) {
    const size_t rows = std::min<size_t>({(avail - want - 256) / row_bytes, (size_t)R * S, 0xffffffffu});
    if (rows >= (size_t)S) {
      L.xcap = (uint32_t)rows;
      xbytes = align256(rows * row_bytes);
      L.xstore = reinterpret_cast<uint4*>(p + ob);
    }
  }
  L.stage = reinterpret_cast<float*>(p + ob + xbytes);
  L.per_round = std::min<int64_t>((int64_t)((avail - xbytes) / per_ray), R);
  if (L.per_round <= 0 || (R + L.per_round - 1) / L.per_round > kMaxStagedRounds) {
    L.per_round = 0;
    L.xstore = nullptr;
    L.xcap = 0;
  }
  return L;
}

// Time slice of a 4D grid at the batch's t (mixed training).  Along t a
// level's 16-corner interpolation is a blend of two time vertices with the
// same weights for every sample of the batch, and the vertices' entries are
// the 3D vertex's entry XOR a per-level constant (hashed levels: the hash is
// an XOR of per-axis terms, masked) or plus a per-level offset (dense levels:
// t is the outermost stride).  So per level
//   slice[k] = w0 * table[k ^ c0] + w1 * table[k ^ c1]   (hashed)
//   slice[k] = w0 * table[k + c0] + w1 * table[k + c1]   (dense, k < x*y*z vertices)
// and the 3D view g3 of the grid (same resolutions, strides and hash, slice
// offsets) indexes it: the 3D kernels then gather 8 corners instead of 16.
// Gradients reduced into a slice-shaped table g are spread back by
//   dtable[e] += w0 * g[e ^ c0] + w1 * g[e ^ c1]          (hashed; conflict-free)
//   dtable[k + c0] += w0 * g[k], dtable[k + c1] += w1 * g[k]  (dense)
struct TimeSlice {
  GridDev g3;
  int64_t off4[NECTB_MAX_LEVELS];    // the 4D level offsets
  int64_t n_real[NECTB_MAX_LEVELS];  // slice entries that exist (T, or the dense x*y*z vertices)
  int64_t c0[NECTB_MAX_LEVELS], c1[NECTB_MAX_LEVELS];
  float w0[NECTB_MAX_LEVELS], w1[NECTB_MAX_LEVELS];
};

// t -> vertex and weights exactly as level_corners computes them for axis 3.
inline TimeSlice make_time_slice(const GridDev& g, float t) {
  TimeSlice s;
  s.g3 = g;
  s.g3.n_dims = 3;
  int64_t off = 0;
  for (int l = 0; l < g.n_levels; ++l) {
    s.off4[l] = g.offset[l];
    const int r = g.res[l][3];
    const float p = t * (float)r;
    int ci = (int)std::floor(p);
    ci = ci < 0 ? 0 : (ci > r - 1 ? r - 1 : ci);
    const float f = p - (float)ci;
    s.w0[l] = 1.f - f;
    s.w1[l] = f;
    const bool hashed = (g.hashed_bits >> l) & 1u;
    if (hashed) {
      const uint32_t term = (uint32_t)ci * kPrime3;
      s.c0[l] = (int64_t)(term & g.hash_mask);
      s.c1[l] = (int64_t)((term + kPrime3) & g.hash_mask);
      s.n_real[l] = (int64_t)g.hash_mask + 1;
    } else {
      const int64_t s3 = g.stride[l][3];
      s.c0[l] = (int64_t)ci * s3;
      s.c1[l] = (int64_t)(ci + 1) * s3;
      s.n_real[l] = s3;
    }
    s.g3.offset[l] = off;
    off += hashed ? s.n_real[l] : (s.n_real[l] + 7) / 8 * 8;
  }
  s.g3.total_entries = off;
  return s;
}

// Bytes of a 4D grid's time slice (fp16) and its fp32 gradient, for one step.
inline size_t slice_bytes(const GridDev& g) {
  const int64_t n3 = make_time_slice(g, 0.f).g3.total_entries;
  return align256((size_t)n3 * g.n_features * 2) + align256((size_t)n3 * g.n_features * 4);
}

// A texture object over an fp16 table (entry_bytes 4 or 8), cached per
// buffer, or 0 where none can be made; the encoders fetch the odd hashed
// levels' corners through it.
cudaTextureObject_t table_texture(const void* ptr, size_t bytes, int entry_bytes);

// Bytes of the fp16 time slice alone (forward-only queries).
inline size_t slice_half_bytes(const GridDev& g) {
  return align256((size_t)make_time_slice(g, 0.f).g3.total_entries * g.n_features * 2);
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
// rounds of equal ray counts: order[rank] = ray, ranks 0..ctrl[6]-1, and
// offs[rank] = samples of the rays ranked before it (the ray's first row in
// the encoding store).  Three launches over the scheduling indices (pixels,
// or batch positions when the batch repeats a pixel): per-block counts, one
// block scanning them, and the per-block compaction, so pixel order is kept.
__global__ void order_count_kernel(const int32_t* __restrict__ slot, const RayRec* __restrict__ recs,
                                   const unsigned int* __restrict__ ctrl, int R, int P,
                                   unsigned int* __restrict__ block_sums,
                                   unsigned long long* __restrict__ block_samples);
__global__ void order_scan_kernel(unsigned int* __restrict__ block_sums, unsigned long long* __restrict__ block_samples,
                                  int n_blocks, unsigned int* __restrict__ ctrl);
__global__ void order_compact_kernel(const int32_t* __restrict__ slot, const RayRec* __restrict__ recs,
                                     const unsigned int* __restrict__ ctrl, int R, int P,
                                     const unsigned int* __restrict__ block_sums,
                                     const unsigned long long* __restrict__ block_samples,
                                     int32_t* __restrict__ order, uint64_t* __restrict__ offs);

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
