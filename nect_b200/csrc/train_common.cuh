// Pieces shared by the plain (fp32 SIMT) and mixed (bf16 tcgen05) fused
// training kernels: per-ray records, the ray-preparation kernel, sample
// regeneration and the workspace layout.
#pragma once
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

struct TrainArgs {
  const int64_t* perm;
  int64_t perm_len;
  int64_t start;
  int num_rays;
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
};

// Workspace: RayRec[R] then two scheduling counters (fwd, bwd) and padding.
struct Workspace {
  RayRec* rays;
  unsigned int* counters;  // [0] forward ray cursor, [1] backward ray cursor
};

inline size_t workspace_bytes(int R) { return (size_t)R * sizeof(RayRec) + 256; }

inline Workspace carve_workspace(void* ws, int R) {
  Workspace w;
  w.rays = (RayRec*)ws;
  w.counters = (unsigned int*)((char*)ws + (size_t)R * sizeof(RayRec));
  return w;
}

// Warp per ray: set-up, sample count (warp ballot), measured value, scale.
__global__ void ray_prep_kernel(NectbGeometry g, TrainArgs a, RayRec* __restrict__ recs);

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

// Loss gradient dL/dy_pred for one ray (mean over rays, nect/config.py:481-497).
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
