// Ray geometry shared by the sampling kernel and the fused training and
// query kernels.
//
// The arithmetic restates the reference sampler expression by expression
// (nect/sampling/ct_sampling.cu:121-576): the same mix of fp32 trigonometry
// and fp64 point arithmetic, the same evaluation order, and the same
// per-axis break tests, so that sample positions and per-ray sample counts
// come out bit-identical to the reference kernel compiled with the same
// nvcc.  Only the organisation differs: the per-ray set-up is a pure function
// of (geometry, pixel, draws), and sample i is a pure function of the set-up,
// so a warp can evaluate 32 samples of a ray at once and a fused kernel can
// regenerate any sample in registers without storing positions.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/nectb.h"

namespace nectb {

struct P3 {
  double x, y, z;
};

// Per-ray state after entry/exit, normalisation, jitter and clamping.
struct RaySetup {
  P3 start;    // first sample, normalised to [0,1]^3 (clamped)
  P3 end;      // exit bound used by the break tests (clamped)
  P3 step;     // sample spacing in normalised coordinates
  float distance;  // distances[tid] of the reference
  int valid;       // 0: ray missed the object (nothing written)
};

__device__ __forceinline__ void rotate_pair(P3& a, P3& b, float angle_rad, float COR) {
  // ct_sampling.cu:121-128
  float cos_angle = cosf(angle_rad);
  float sin_angle = sinf(angle_rad);
  a.y = a.y - COR;
  b.y = b.y - COR;
  P3 na = {cos_angle * a.x - sin_angle * a.y, sin_angle * a.x + cos_angle * a.y, a.z};
  P3 nb = {cos_angle * b.x - sin_angle * b.y, sin_angle * b.x + cos_angle * b.y, b.z};
  a = na;
  b = nb;
}

__device__ __forceinline__ double dmax_std(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin_std(double a, double b) { return (b < a) ? b : a; }

// Slab test against the box [lo, hi] for the segment a->b (fp64),
// ct_sampling.cu:160-198.
__device__ __forceinline__ bool segment_box(P3 a, P3 b, P3 lo, P3 hi, P3& p, P3& q) {
  double tx0 = (lo.x - a.x) / (b.x - a.x);
  double tx1 = (hi.x - a.x) / (b.x - a.x);
  if (tx0 > tx1) { double t = tx0; tx0 = tx1; tx1 = t; }
  double ty0 = (lo.y - a.y) / (b.y - a.y);
  double ty1 = (hi.y - a.y) / (b.y - a.y);
  if (ty0 > ty1) { double t = ty0; ty0 = ty1; ty1 = t; }
  double tz0 = (lo.z - a.z) / (b.z - a.z);
  double tz1 = (hi.z - a.z) / (b.z - a.z);
  if (tz0 > tz1) { double t = tz0; tz0 = tz1; tz1 = t; }
  double tmin = dmax_std(dmax_std(tx0, ty0), tz0);
  double tmax = dmin_std(dmin_std(tx1, ty1), tz1);
  if (tmin > tmax || !(tmin >= 0.0 && tmin <= 1.0) || !(tmax >= 0.0 && tmax <= 1.0)) return false;
  p.x = a.x + tmin * (b.x - a.x);
  p.y = a.y + tmin * (b.y - a.y);
  p.z = a.z + tmin * (b.z - a.z);
  q.x = a.x + tmax * (b.x - a.x);
  q.y = a.y + tmax * (b.y - a.y);
  q.z = a.z + tmax * (b.z - a.z);
  return true;
}

// Detector tilt (roll, pitch, yaw), ct_sampling.cu:200-224.
__device__ __forceinline__ void tilt_detector(const NectbGeometry& g, P3& p) {
  float alpha_ = g.rotDetector[2];
  float beta_ = g.rotDetector[1];
  float gamma_ = g.rotDetector[0];
  float c_alpha = cosf(-alpha_);
  float c_beta = cosf(-beta_);
  float c_gamma = cosf(-gamma_);
  float s_alpha = sinf(-alpha_);
  float s_beta = sinf(-beta_);
  float s_gamma = sinf(-gamma_);
  float R12 = c_alpha * s_beta * s_gamma - s_alpha * c_gamma;
  float R13 = c_alpha * s_beta * c_gamma + s_alpha * s_gamma;
  float R22 = s_alpha * s_beta * s_gamma + c_alpha * c_gamma;
  float R23 = s_alpha * s_beta * c_gamma - c_alpha * s_gamma;
  float R32 = c_beta * s_gamma;
  float R33 = c_beta * c_gamma;
  float x = R12 * p.y + R13 * p.z;
  float y = R22 * p.y + R23 * p.z;
  float z = R32 * p.y + R33 * p.z;
  p.x = x;
  p.y = y;
  p.z = z;
}

// Detector pixel position for a flat detector at x = 0, ct_sampling.cu:226-245.
__device__ __forceinline__ void pixel_position(const NectbGeometry& g, int ray_index, float off0,
                                               float off1, P3& p) {
  int col = ray_index % g.nDetector[1];
  int row = ray_index / g.nDetector[1];
  float detector_xy = (col - (static_cast<float>(g.nDetector[1] - 1) / 2) + off0) * g.dDetector[1] + g.offDetector[1];
  p.y = -detector_xy;
  p.z = (row - (static_cast<float>(g.nDetector[0] - 1) / 2) + off1) * g.dDetector[0] + g.offDetector[0];
  p.x = 0;
  if (g.rotDetector[0] != 0 || g.rotDetector[1] != 0 || g.rotDetector[2] != 0) tilt_detector(g, p);
}

// Ray/cylinder entry and exit, ct_sampling.cu:258-288.
__device__ __forceinline__ bool cylinder_entry_exit(const NectbGeometry& g, P3 p1, P3 dir, float angle_rad,
                                                    P3& s, P3& e) {
  float a = dir.x * dir.x + dir.y * dir.y;
  float b = 2 * p1.x * dir.x + 2 * (p1.y - g.COR) * dir.y;
  float c = p1.x * p1.x + p1.y * p1.y - g.object_radius * g.object_radius;
  float discriminant = b * b - 4 * a * c;
  if (discriminant <= 0) return false;
  float sqrt_discriminant = sqrtf(discriminant);
  float two_a = 2 * a;
  float t1 = (-b - sqrt_discriminant) / (two_a);
  float t2 = (-b + sqrt_discriminant) / (two_a);
  s.x = (p1.x + t1 * dir.x);
  s.y = (p1.y + t1 * dir.y);
  s.z = (t1 * dir.z);
  e.x = (p1.x + t2 * dir.x);
  e.y = (p1.y + t2 * dir.y);
  e.z = (t2 * dir.z);
  rotate_pair(s, e, angle_rad, g.COR);
  return true;
}

// Entry/exit of one ray in world units (calc_start_end_points,
// ct_sampling.cu:290-389).  Returns false when the ray misses.
__device__ __forceinline__ bool entry_exit(const NectbGeometry& g, int ray_index, float off0, float off1,
                                           float angle_rad, P3& s, P3& e) {
  switch (g.kind) {
    case NECTB_CONE_VOXEL: {
      P3 p1 = {-(double)g.distance_source_to_origin, 0, 0};
      P3 p2;
      pixel_position(g, ray_index, off0, off1, p2);
      p2.x = p2.x + g.distance_origin_to_detector;
      rotate_pair(p1, p2, angle_rad, g.COR);
      float sX = (g.sVoxel[2] - g.dVoxel[2] / 2) / 2;
      float sY = (g.sVoxel[1] - g.dVoxel[1] / 2) / 2;
      float sZ = (g.sVoxel[0] - g.dVoxel[0] / 2) / 2;
      P3 lo = {-sX, -sY, -sZ};
      P3 hi = {sX, sY, sZ};
      return segment_box(p1, p2, lo, hi, s, e);
    }
    case NECTB_PARALLEL_VOXEL: {
      P3 p2;
      pixel_position(g, ray_index, off0, off1, p2);
      p2.x = p2.x + sqrtf(g.sVoxel[2] * g.sVoxel[2] + g.sVoxel[1] * g.sVoxel[1]);
      P3 p1 = {-p2.x, p2.y, p2.z};
      rotate_pair(p1, p2, angle_rad, g.COR);
      float sX = (g.sVoxel[2] - g.dVoxel[2] / 2) / 2;
      float sY = (g.sVoxel[1] - g.dVoxel[1] / 2) / 2;
      float sZ = (g.sVoxel[0] - g.dVoxel[0] / 2) / 2;
      P3 lo = {-sX, -sY, -sZ};
      P3 hi = {sX, sY, sZ};
      return segment_box(p1, p2, lo, hi, s, e);
    }
    case NECTB_CONE_CYLINDRICAL: {
      P3 p1 = {-(double)g.distance_source_to_origin, 0, 0};
      P3 p2;
      pixel_position(g, ray_index, off0, off1, p2);
      p2.x = p2.x + g.distance_origin_to_detector;
      P3 dir = {p2.x - p1.x, p2.y, p2.z};
      return cylinder_entry_exit(g, p1, dir, angle_rad, s, e);
    }
    case NECTB_PARALLEL_CYLINDRICAL: {
      P3 p2;
      pixel_position(g, ray_index, off0, off1, p2);
      p2.x = p2.x + g.object_radius;
      P3 p1 = {-p2.x, p2.y, p2.z};
      P3 dir = {p2.x - p1.x, 0, 0};
      return cylinder_entry_exit(g, p1, dir, angle_rad, s, e);
    }
    default:
      return false;
  }
}

__device__ __forceinline__ double clamp01(double v) { return fmin(fmax(v, (double)0.0f), (double)1.0f); }

// Normalisation, spacing, jitter and clamping (calc_all_points before its
// loop: voxel ct_sampling.cu:486-530, cylindrical :402-437).
__device__ __forceinline__ void finish_setup(const NectbGeometry& g, P3 s, P3 e, int S, float maxd, bool uniform,
                                             float jit, RaySetup& r) {
  P3 step = {e.x - s.x, e.y - s.y, e.z - s.z};
  float ray_distance = sqrt(step.x * step.x + step.y * step.y + step.z * step.z);
  const bool voxel = (g.kind == NECTB_CONE_VOXEL || g.kind == NECTB_PARALLEL_VOXEL);
  if (voxel) {
    if (uniform) {
      r.distance = maxd;
      step.x = (step.x / ray_distance) * maxd / g.sVoxel[2];
      step.y = (step.y / ray_distance) * maxd / g.sVoxel[1];
      step.z = (step.z / ray_distance) * maxd / g.sVoxel[0];
    } else {
      r.distance = ray_distance / S;
      step.x = (step.x / S) / g.sVoxel[2];
      step.y = (step.y / S) / g.sVoxel[1];
      step.z = (step.z / S) / g.sVoxel[0];
    }
    s.x /= (g.sVoxel[2]);
    e.x /= (g.sVoxel[2]);
    s.y /= (g.sVoxel[1]);
    e.y /= (g.sVoxel[1]);
    s.z /= (g.sVoxel[0]);
    e.z /= (g.sVoxel[0]);
    P3 ns = {s.x + 0.5 + jit * step.x, s.y + 0.5 + jit * step.y, s.z + 0.5 + jit * step.z};
    P3 ne = {e.x + 0.5 + step.x, e.y + 0.5 + step.y, e.z + 0.5 + step.z};
    s = ns;
    e = ne;
  } else {
    if (uniform) {
      r.distance = maxd;
      step.x = (step.x / ray_distance) * maxd / (2 * g.object_radius);
      step.y = (step.y / ray_distance) * maxd / (2 * g.object_radius);
      step.z = (step.z / ray_distance) * maxd / (g.object_height);
    } else {
      r.distance = ray_distance / S;
      step.x = (step.x / S) / (2 * g.object_radius);
      step.y = (step.y / S) / (2 * g.object_radius);
      step.z = (step.z / S) / (g.object_height);
    }
    s.x /= 2 * g.object_radius;
    e.x /= 2 * g.object_radius;
    s.y /= 2 * g.object_radius;
    e.y /= 2 * g.object_radius;
    s.z /= (g.object_height);
    P3 ns = {s.x + 0.5 + jit * step.x, s.y + 0.5 + jit * step.y, s.z + 0.5 + jit * step.z};
    P3 ne = {e.x + 0.5, e.y + 0.5, e.z};
    s = ns;
    e = ne;
  }
  s.z = clamp01(s.z);
  s.y = clamp01(s.y);
  s.x = clamp01(s.x);
  e.z = clamp01(e.z);
  e.y = clamp01(e.y);
  e.x = clamp01(e.x);
  r.start = s;
  r.end = e;
  r.step = step;
}

// Full per-ray set-up.  Returns false (r.valid = 0) when the reference kernel
// would return before writing anything for this ray.
__device__ __forceinline__ bool ray_setup(const NectbGeometry& g, int ray_index, float off0, float off1, float jit,
                                          float angle_rad, int S, float maxd, bool uniform, RaySetup& r) {
  P3 s, e;
  r.valid = 0;
  r.distance = 0.f;
  if (!entry_exit(g, ray_index, off0, off1, angle_rad, s, e)) return false;
  finish_setup(g, s, e, S, maxd, uniform, jit, r);
  r.valid = 1;
  return true;
}

// Sample i of a set-up ray: position (unclamped fp32, z,y,x) and whether the
// reference loop would break at i (ct_sampling.cu:537-575 voxel,
// :440-472 cylindrical).
__device__ __forceinline__ bool sample_at(const NectbGeometry& g, const RaySetup& r, int i, float& pz, float& py,
                                          float& px) {
  float pos_x = r.start.x + i * r.step.x;
  float pos_y = r.start.y + i * r.step.y;
  float pos_z = r.start.z + i * r.step.z;
  pz = pos_z;
  py = pos_y;
  px = pos_x;
  const bool voxel = (g.kind == NECTB_CONE_VOXEL || g.kind == NECTB_PARALLEL_VOXEL);
  if (voxel) {
    const float eps = 1e-5f;
    if (r.step.x > 0) {
      if (pos_x - eps > r.end.x) return false;
    } else if (r.step.x < 0) {
      if (pos_x + eps < r.end.x) return false;
    }
    if (r.step.y > 0) {
      if (pos_y - eps > r.end.y) return false;
    } else if (r.step.y < 0) {
      if (pos_y + eps < r.end.y) return false;
    }
    if (r.step.z > 0) {
      if (pos_z - eps > r.end.z) return false;
    } else if (r.step.z < 0) {
      if (pos_z + eps < r.end.z) return false;
    }
    return true;
  }
  if (r.step.x > 0) {
    if (pos_x > r.end.x) return false;
  } else if (r.step.x < 0) {
    if (pos_x < r.end.x) return false;
  } else if (r.step.y > 0) {
    if (pos_y > r.end.y) return false;
  } else if (r.step.y < 0) {
    if (pos_y < r.end.y) return false;
  }
  if (pos_z < 0 + g.remove_factor_top || pos_z > 1 - g.remove_factor_bottom) return false;
  return true;
}

// Projector clamp (projector.py:127) of a position that the sampler wrote.
__device__ __forceinline__ float clamp01f(float v) { return fminf(fmaxf(v, 0.f), 1.f); }

// Ray index lookup with the reference's bounds checks (ct_sampling.cu:130-148).
__device__ __forceinline__ bool ray_lookup(const int64_t* perm, int64_t perm_len, int64_t start, int tid,
                                           int num_rays, const NectbGeometry& g, int& ray_index) {
  if (tid >= num_rays) return false;
  if (tid + start >= perm_len) return false;
  ray_index = (int)perm[tid + start];
  if (ray_index >= g.nDetector[0] * g.nDetector[1]) return false;
  return true;
}

// Warp-cooperative count of written samples: the first i in [0,S) at which
// the reference loop breaks (S when it never does).  All 32 lanes must call.
__device__ __forceinline__ int warp_sample_count(const NectbGeometry& g, const RaySetup& r, int S, int lane) {
  for (int base = 0; base < S; base += 32) {
    int i = base + lane;
    bool ok = true;
    if (i < S) {
      float a, b, c;
      ok = sample_at(g, r, i, a, b, c);
    }
    unsigned fail = __ballot_sync(0xffffffffu, !ok);
    if (fail) {
      int first = base + __ffs(fail) - 1;
      return first < S ? first : S;
    }
  }
  return S;
}

}  // namespace nectb
