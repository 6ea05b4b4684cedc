/*
 * CPU oracle for the ray sampler.  TEST INFRASTRUCTURE ONLY: imported by
 * tests/, __graft_entry__.smoke() and the cpu_baseline / reference arm of
 * bench.py, never by the product path.
 *
 * A plain-C restatement of the reference sampler
 * nect/sampling/ct_sampling.cu (haakonnese/nect):
 *   rotate_points            :121-128   -> rotate_pair
 *   get_tid_ray_index        :130-148   -> ray_lookup
 *   findIntersection         :160-198   -> segment_box
 *   rotate_detector          :200-224   -> tilt_detector
 *   calc_xyz_detector_pos*   :226-256   -> pixel_position
 *   start_end_helper         :258-288   -> cylinder_entry_exit
 *   calc_start_end_points    :290-389   -> entry_exit
 *   calc_all_points          :392-576   -> finish_setup + sample_at
 *   sample_points / sample   :578-648   -> oracle_sample
 * with the reference's fp32/fp64 mix and evaluation order.  The device
 * compiler contracts multiply-add pairs into FMAs; the host build disables
 * contraction (-ffp-contract=off) and writes the contractions out with fma()
 * where a multiply feeds an add, so host results can be compared bit for bit
 * with the device.  Device cosf/sinf may differ from the host libm by an ulp,
 * so callers may pass the device's trig values (trig[8], see oracle_trig).
 * Parity is pinned by tests/golden/sampling_golden.npz, produced by running
 * the reference kernel itself (tests/golden/make_sampling_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../include/nectb.h"

typedef struct {
  double x, y, z;
} P3;

typedef struct {
  P3 start, end, step;
  float distance;
  int valid;
} RaySetup;

/* trig[0..1] = cos, sin of the projection angle; trig[2..7] = cos(-yaw),
 * cos(-pitch), cos(-roll), sin(-yaw), sin(-pitch), sin(-roll). */
void oracle_trig(const NectbGeometry* g, float angle, float* trig) {
  trig[0] = cosf(angle);
  trig[1] = sinf(angle);
  trig[2] = cosf(-g->rotDetector[2]);
  trig[3] = cosf(-g->rotDetector[1]);
  trig[4] = cosf(-g->rotDetector[0]);
  trig[5] = sinf(-g->rotDetector[2]);
  trig[6] = sinf(-g->rotDetector[1]);
  trig[7] = sinf(-g->rotDetector[0]);
}

static void rotate_pair(P3* a, P3* b, const float* trig, float COR) {
  double c = (double)trig[0], s = (double)trig[1];
  a->y = a->y - COR;
  b->y = b->y - COR;
  P3 na = {fma(c, a->x, -(s * a->y)), fma(s, a->x, c * a->y), a->z};
  P3 nb = {fma(c, b->x, -(s * b->y)), fma(s, b->x, c * b->y), b->z};
  *a = na;
  *b = nb;
}

static double dmax_std(double a, double b) { return (a < b) ? b : a; }
static double dmin_std(double a, double b) { return (b < a) ? b : a; }

static int segment_box(P3 a, P3 b, P3 lo, P3 hi, P3* p, P3* q) {
  double tx0 = (lo.x - a.x) / (b.x - a.x), tx1 = (hi.x - a.x) / (b.x - a.x);
  if (tx0 > tx1) { double t = tx0; tx0 = tx1; tx1 = t; }
  double ty0 = (lo.y - a.y) / (b.y - a.y), ty1 = (hi.y - a.y) / (b.y - a.y);
  if (ty0 > ty1) { double t = ty0; ty0 = ty1; ty1 = t; }
  double tz0 = (lo.z - a.z) / (b.z - a.z), tz1 = (hi.z - a.z) / (b.z - a.z);
  if (tz0 > tz1) { double t = tz0; tz0 = tz1; tz1 = t; }
  double tmin = dmax_std(dmax_std(tx0, ty0), tz0);
  double tmax = dmin_std(dmin_std(tx1, ty1), tz1);
  if (tmin > tmax || !(tmin >= 0.0 && tmin <= 1.0) || !(tmax >= 0.0 && tmax <= 1.0)) return 0;
  p->x = fma(tmin, b.x - a.x, a.x);
  p->y = fma(tmin, b.y - a.y, a.y);
  p->z = fma(tmin, b.z - a.z, a.z);
  q->x = fma(tmax, b.x - a.x, a.x);
  q->y = fma(tmax, b.y - a.y, a.y);
  q->z = fma(tmax, b.z - a.z, a.z);
  return 1;
}

static void tilt_detector(const float* trig, P3* p) {
  float c_alpha = trig[2], c_beta = trig[3], c_gamma = trig[4];
  float s_alpha = trig[5], s_beta = trig[6], s_gamma = trig[7];
  float cs = c_alpha * s_beta, ss = s_alpha * s_beta;
  float R12 = fmaf(cs, s_gamma, -(s_alpha * c_gamma));
  float R13 = fmaf(cs, c_gamma, s_alpha * s_gamma);
  float R22 = fmaf(ss, s_gamma, c_alpha * c_gamma);
  float R23 = fmaf(ss, c_gamma, -(c_alpha * s_gamma));
  float R32 = c_beta * s_gamma;
  float R33 = c_beta * c_gamma;
  float x = (float)fma((double)R12, p->y, (double)R13 * p->z);
  float y = (float)fma((double)R22, p->y, (double)R23 * p->z);
  float z = (float)fma((double)R32, p->y, (double)R33 * p->z);
  p->x = x;
  p->y = y;
  p->z = z;
}

static void pixel_position(const NectbGeometry* g, int ray_index, float off0, float off1, const float* trig, P3* p) {
  int col = ray_index % g->nDetector[1];
  int row = ray_index / g->nDetector[1];
  float a = (float)col - ((float)(g->nDetector[1] - 1) / 2.0f) + off0;
  float xy = fmaf(a, g->dDetector[1], g->offDetector[1]);
  p->y = -xy;
  float b = (float)row - ((float)(g->nDetector[0] - 1) / 2.0f) + off1;
  p->z = fmaf(b, g->dDetector[0], g->offDetector[0]);
  p->x = 0;
  if (g->rotDetector[0] != 0 || g->rotDetector[1] != 0 || g->rotDetector[2] != 0) tilt_detector(trig, p);
}

static int cylinder_entry_exit(const NectbGeometry* g, P3 p1, P3 dir, const float* trig, P3* s, P3* e) {
  float a = (float)fma(dir.x, dir.x, dir.y * dir.y);
  float b = (float)fma(2 * p1.x, dir.x, (2 * (p1.y - g->COR)) * dir.y);
  float c = (float)(fma(p1.x, p1.x, p1.y * p1.y) - (double)(g->object_radius * g->object_radius));
  float disc = fmaf(b, b, -((4 * a) * c));
  if (disc <= 0) return 0;
  float sq = sqrtf(disc);
  float two_a = 2 * a;
  float t1 = (-b - sq) / two_a;
  float t2 = (-b + sq) / two_a;
  s->x = fma((double)t1, dir.x, p1.x);
  s->y = fma((double)t1, dir.y, p1.y);
  s->z = (double)t1 * dir.z;
  e->x = fma((double)t2, dir.x, p1.x);
  e->y = fma((double)t2, dir.y, p1.y);
  e->z = (double)t2 * dir.z;
  rotate_pair(s, e, trig, g->COR);
  return 1;
}

static int entry_exit(const NectbGeometry* g, int ray_index, float off0, float off1, const float* trig, P3* s,
                      P3* e) {
  P3 p1, p2;
  switch (g->kind) {
    case NECTB_CONE_VOXEL:
    case NECTB_PARALLEL_VOXEL: {
      pixel_position(g, ray_index, off0, off1, trig, &p2);
      if (g->kind == NECTB_CONE_VOXEL) {
        p1.x = -(double)g->distance_source_to_origin;
        p1.y = 0;
        p1.z = 0;
        p2.x = p2.x + g->distance_origin_to_detector;
      } else {
        p2.x = p2.x + sqrtf(fmaf(g->sVoxel[2], g->sVoxel[2], g->sVoxel[1] * g->sVoxel[1]));
        p1.x = -p2.x;
        p1.y = p2.y;
        p1.z = p2.z;
      }
      rotate_pair(&p1, &p2, trig, g->COR);
      float sX = (g->sVoxel[2] - g->dVoxel[2] / 2) / 2;
      float sY = (g->sVoxel[1] - g->dVoxel[1] / 2) / 2;
      float sZ = (g->sVoxel[0] - g->dVoxel[0] / 2) / 2;
      P3 lo = {-sX, -sY, -sZ}, hi = {sX, sY, sZ};
      return segment_box(p1, p2, lo, hi, s, e);
    }
    case NECTB_CONE_CYLINDRICAL: {
      p1.x = -(double)g->distance_source_to_origin;
      p1.y = 0;
      p1.z = 0;
      pixel_position(g, ray_index, off0, off1, trig, &p2);
      p2.x = p2.x + g->distance_origin_to_detector;
      P3 dir = {p2.x - p1.x, p2.y, p2.z};
      return cylinder_entry_exit(g, p1, dir, trig, s, e);
    }
    case NECTB_PARALLEL_CYLINDRICAL: {
      pixel_position(g, ray_index, off0, off1, trig, &p2);
      p2.x = p2.x + g->object_radius;
      p1.x = -p2.x;
      p1.y = p2.y;
      p1.z = p2.z;
      P3 dir = {p2.x - p1.x, 0, 0};
      return cylinder_entry_exit(g, p1, dir, trig, s, e);
    }
  }
  return 0;
}

static double clamp01(double v) { return fmin(fmax(v, 0.0), 1.0); }

static void finish_setup(const NectbGeometry* g, P3 s, P3 e, int S, float maxd, int uniform, float jit, RaySetup* r) {
  P3 st = {e.x - s.x, e.y - s.y, e.z - s.z};
  float ray_distance = (float)sqrt(fma(st.z, st.z, fma(st.x, st.x, st.y * st.y)));
  int voxel = (g->kind == NECTB_CONE_VOXEL || g->kind == NECTB_PARALLEL_VOXEL);
  double sx, sy, sz;
  if (voxel) {
    sx = g->sVoxel[2];
    sy = g->sVoxel[1];
    sz = g->sVoxel[0];
  } else {
    sx = (double)(2 * g->object_radius);
    sy = sx;
    sz = g->object_height;
  }
  if (uniform) {
    r->distance = maxd;
    st.x = (st.x / ray_distance) * maxd / sx;
    st.y = (st.y / ray_distance) * maxd / sy;
    st.z = (st.z / ray_distance) * maxd / sz;
  } else {
    r->distance = ray_distance / (float)S;
    st.x = (st.x / S) / sx;
    st.y = (st.y / S) / sy;
    st.z = (st.z / S) / sz;
  }
  s.x /= sx;
  e.x /= sx;
  s.y /= sy;
  e.y /= sy;
  s.z /= sz;
  double jd = (double)jit;
  P3 ns = {fma(jd, st.x, s.x + 0.5), fma(jd, st.y, s.y + 0.5), fma(jd, st.z, s.z + 0.5)};
  P3 ne;
  if (voxel) {
    e.z /= sz;
    ne.x = e.x + 0.5 + st.x;
    ne.y = e.y + 0.5 + st.y;
    ne.z = e.z + 0.5 + st.z;
  } else {
    ne.x = e.x + 0.5;
    ne.y = e.y + 0.5;
    ne.z = e.z; /* the reference does not normalise or shift end.z here */
  }
  r->start.x = clamp01(ns.x);
  r->start.y = clamp01(ns.y);
  r->start.z = clamp01(ns.z);
  r->end.x = clamp01(ne.x);
  r->end.y = clamp01(ne.y);
  r->end.z = clamp01(ne.z);
  r->step = st;
}

static int sample_at(const NectbGeometry* g, const RaySetup* r, int i, float* pz, float* py, float* px) {
  double di = (double)i;
  float pos_x = (float)fma(di, r->step.x, r->start.x);
  float pos_y = (float)fma(di, r->step.y, r->start.y);
  float pos_z = (float)fma(di, r->step.z, r->start.z);
  *pz = pos_z;
  *py = pos_y;
  *px = pos_x;
  if (g->kind == NECTB_CONE_VOXEL || g->kind == NECTB_PARALLEL_VOXEL) {
    const float eps = 1e-5f;
    if (r->step.x > 0) {
      if ((double)(pos_x - eps) > r->end.x) return 0;
    } else if (r->step.x < 0) {
      if ((double)(pos_x + eps) < r->end.x) return 0;
    }
    if (r->step.y > 0) {
      if ((double)(pos_y - eps) > r->end.y) return 0;
    } else if (r->step.y < 0) {
      if ((double)(pos_y + eps) < r->end.y) return 0;
    }
    if (r->step.z > 0) {
      if ((double)(pos_z - eps) > r->end.z) return 0;
    } else if (r->step.z < 0) {
      if ((double)(pos_z + eps) < r->end.z) return 0;
    }
    return 1;
  }
  if (r->step.x > 0) {
    if (pos_x > r->end.x) return 0;
  } else if (r->step.x < 0) {
    if (pos_x < r->end.x) return 0;
  } else if (r->step.y > 0) {
    if (pos_y > r->end.y) return 0;
  } else if (r->step.y < 0) {
    if (pos_y < r->end.y) return 0;
  }
  if (pos_z < 0 + g->remove_factor_top || pos_z > 1 - g->remove_factor_bottom) return 0;
  return 1;
}

/* One ray: fills out[S*3] (or only the count when out is NULL) and returns
 * the number of written samples; *distance receives distances[tid]. */
int oracle_ray(const NectbGeometry* g, int ray_index, float off0, float off1, float jit, const float* trig, int S,
               float maxd, int uniform, float* out, float* distance) {
  P3 s, e;
  RaySetup r;
  *distance = 0.f;
  if (out) memset(out, 0, sizeof(float) * 3 * (size_t)S);
  if (!entry_exit(g, ray_index, off0, off1, trig, &s, &e)) return 0;
  finish_setup(g, s, e, S, maxd, uniform, jit, &r);
  *distance = r.distance;
  int n = 0;
  for (int i = 0; i < S; i++) {
    float pz, py, px;
    if (!sample_at(g, &r, i, &pz, &py, &px)) break;
    if (out) {
      out[3 * i + 0] = pz;
      out[3 * i + 1] = py;
      out[3 * i + 2] = px;
    }
    n++;
  }
  return n;
}

/* Batch entry with the reference's bounds checks; trig may be NULL (host
 * libm values are used then).  Returns 0. */
int oracle_sample(const NectbGeometry* g, const int64_t* perm, int64_t perm_len, int64_t start, int num_rays, int S,
                  float angle, float maxd, int uniform, const float* jitter, const float* det_off, const float* trig,
                  float* points, float* distances, int32_t* counts) {
  float own[8];
  if (!trig) {
    oracle_trig(g, angle, own);
    trig = own;
  }

  for (int tid = 0; tid < num_rays; tid++) {
    float* out = points ? points + (size_t)tid * S * 3 : 0;
    float dist = 0.f;
    int n = 0;
    int valid = (tid + start < perm_len);
    int ray_index = valid ? (int)perm[tid + start] : 0;
    if (valid && ray_index >= g->nDetector[0] * g->nDetector[1]) valid = 0;
    if (valid) {
      n = oracle_ray(g, ray_index, det_off[2 * tid], det_off[2 * tid + 1], jitter[tid], trig, S, maxd, uniform, out,
                     &dist);
    } else if (out) {
      memset(out, 0, sizeof(float) * 3 * (size_t)S);
    }
    distances[tid] = dist;
    if (counts) counts[tid] = n;
  }
  return 0;
}
