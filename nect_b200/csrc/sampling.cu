// Ray sampling kernel: the drop-in for the reference's sample_points<T>
// (nect/sampling/ct_sampling.cu:578-602) and host sample<T> (:606-648).
//
// One warp per ray instead of one thread per ray: lanes evaluate 32
// consecutive samples at a time, so the [R,S,3] output is written in
// contiguous 384-byte runs and the zero fill of unwritten samples happens in
// the same pass (the reference first memsets the whole tensor).  The break
// index (= per-ray sample count) is found with a warp ballot.
#include "common.cuh"
#include "geometry.cuh"

namespace nectb {

namespace {

constexpr int kWarpsPerBlock = 8;

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
sample_kernel(NectbGeometry g, const int64_t* __restrict__ perm, int64_t perm_len, int64_t start, int num_rays,
              int S, float angle, float maxd, int uniform, const float* __restrict__ jitter,
              const float* __restrict__ det_off, float* __restrict__ points, float* __restrict__ distances,
              int32_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int tid = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (tid >= num_rays) return;
  int ray_index = 0;
  RaySetup r;
  r.valid = 0;
  r.distance = 0.f;
  if (ray_lookup(perm, perm_len, start, tid, num_rays, g, ray_index)) {
    ray_setup(g, ray_index, det_off[2 * (int64_t)tid], det_off[2 * (int64_t)tid + 1], jitter[tid], angle, S, maxd,
              uniform != 0, r);
  }
  int count = 0;
  if (r.valid) count = warp_sample_count(g, r, S, lane);
  if (lane == 0) {
    distances[tid] = r.distance;
    if (counts) counts[tid] = count;
  }
  if (!points) return;
  float* out = points + (int64_t)tid * S * 3;
  for (int i = lane; i < S; i += 32) {
    float pz = 0.f, py = 0.f, px = 0.f;
    if (i < count) sample_at(g, r, i, pz, py, px);
    out[3 * i + 0] = pz;
    out[3 * i + 1] = py;
    out[3 * i + 2] = px;
  }
}

}  // namespace

int validate_geometry(const NectbGeometry* g) {
  NECTB_REQUIRE(g != nullptr, "geometry is null");
  NECTB_REQUIRE(g->kind >= NECTB_CONE_VOXEL && g->kind <= NECTB_PARALLEL_CYLINDRICAL, "unknown geometry kind %d",
                g->kind);
  NECTB_REQUIRE(g->nDetector[0] > 0 && g->nDetector[1] > 0, "nDetector must be positive");
  NECTB_REQUIRE((int64_t)g->nDetector[0] * g->nDetector[1] <= INT32_MAX, "nDetector has more than 2^31 - 1 pixels");
  return NECTB_OK;
}

}  // namespace nectb

extern "C" int nectb_sample(const NectbGeometry* geometry, const int64_t* random_ray_index,
                            int64_t random_ray_index_len, int64_t starting_ray_index, int32_t num_rays,
                            int32_t num_points_per_ray, float angle_rad, float max_ray_distance_per_point,
                            int32_t uniform_ray_spacing, const float* jitter, const float* detector_offset,
                            float* points, float* distances, int32_t* counts, void* stream) {
  using namespace nectb;
  clear_error();
  if (int rc = validate_geometry(geometry)) return rc;
  NECTB_REQUIRE(num_rays >= 0 && num_points_per_ray >= 0, "negative sizes");
  if (num_rays == 0) return NECTB_OK;
  NECTB_REQUIRE(random_ray_index && jitter && detector_offset && distances, "null input/output pointer");
  NECTB_REQUIRE((int64_t)num_rays * num_points_per_ray * 3 < (int64_t(1) << 40), "points tensor too large");
  const int blocks = (int)ceil_div(num_rays, 8);
  ProfScope ps(kProfSample, (cudaStream_t)stream);
  sample_kernel<<<blocks, 8 * 32, 0, (cudaStream_t)stream>>>(
      *geometry, random_ray_index, random_ray_index_len, starting_ray_index, num_rays, num_points_per_ray, angle_rad,
      max_ray_distance_per_point, uniform_ray_spacing, jitter, detector_offset, points, distances, counts);
  return launch_status("sample_kernel");
}
