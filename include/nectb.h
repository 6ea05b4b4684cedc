/*
 * nectb.h - C ABI of the B200-native NeCT hot path (libnectb.so).
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * (passed as void*), returns an int status (0 = NECTB_OK) and never allocates
 * device memory: callers own every buffer, including workspaces whose sizes the
 * *_workspace_bytes() queries report.  Nothing here synchronises the device;
 * work is ordered on the given stream.  A failed call leaves a message that
 * nectb_last_error() returns (thread-local).
 *
 * Reference interfaces each entry point replaces are cited as
 * path:line within the haakonnese/nect source tree.
 */
#ifndef NECTB_H_
#define NECTB_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  NECTB_OK = 0,
  NECTB_ERR_INVALID = 1,   /* bad argument (null pointer, size, mode)     */
  NECTB_ERR_CUDA = 2,      /* a CUDA launch or runtime call failed         */
  NECTB_ERR_WORKSPACE = 3, /* workspace smaller than *_workspace_bytes()   */
  NECTB_ERR_TOO_LARGE = 4  /* size beyond a documented maximum             */
};

/* ---- geometry ---------------------------------------------------------- */
/* Geometry kinds: the four C++ structs the reference binds
 * (nect/sampling/ct_sampling.cu:7-115, bindings :650-749). */
enum {
  NECTB_CONE_VOXEL = 0,
  NECTB_CONE_CYLINDRICAL = 1,
  NECTB_PARALLEL_VOXEL = 2,
  NECTB_PARALLEL_CYLINDRICAL = 3
};

/* Flat mirror of the reference geometry structs.  Field meaning and units
 * are those of nect/sampling/ct_sampling.cu:7-115; tuples keep their order
 * (nDetector = (rows, cols); sVoxel/dVoxel = (z, y, x); rotDetector =
 * (roll, pitch, yaw)).  Fields a kind does not use are ignored. */
typedef struct NectbGeometry {
  int32_t kind;
  int32_t nDetector[2];
  float dDetector[2];
  float offOrigin[3];
  float offDetector[2];
  float rotDetector[3];
  float COR;
  float distance_source_to_origin;   /* cone kinds */
  float distance_origin_to_detector; /* cone kinds */
  float sVoxel[3];                   /* voxel kinds */
  float dVoxel[3];                   /* voxel kinds */
  float object_radius;               /* cylindrical kinds */
  float object_height;
  float remove_factor_top;
  float remove_factor_bottom;
} NectbGeometry;

/* Ray sampling; replaces sample<T> (nect/sampling/ct_sampling.cu:606-648)
 * and its kernel sample_points<T> (:578-602).  The two random draws the
 * reference makes inside the call (:619-622) are inputs here:
 *   jitter[num_rays]             = U[0,1) - 0.5       (per-ray start offset)
 *   detector_offset[num_rays*2]  = (U[0,1) - 0.5) * random_detector_offset
 * Outputs: points[num_rays*S*3] fp32 in (z,y,x) order with unwritten samples
 * exactly 0 (the kernel writes the zeros; no memset is needed), distances
 * [num_rays] fp32, and optionally counts[num_rays] int32 = samples written per
 * ray (may be NULL).  points may be NULL to compute only distances/counts. */
int nectb_sample(const NectbGeometry* geometry, const int64_t* random_ray_index,
                 int64_t random_ray_index_len, int64_t starting_ray_index,
                 int32_t num_rays, int32_t num_points_per_ray, float angle_rad,
                 float max_ray_distance_per_point, int32_t uniform_ray_spacing,
                 const float* jitter, const float* detector_offset,
                 float* points, float* distances, int32_t* counts, void* stream);

/* ---- hash grid + MLP model -------------------------------------------- */
enum { NECTB_F32 = 0, NECTB_F16 = 1, NECTB_BF16 = 2 };
enum {
  NECTB_ACT_NONE = 0,
  NECTB_ACT_RELU = 1,
  NECTB_ACT_LEAKY_RELU = 2,
  NECTB_ACT_SOFTPLUS = 3,
  NECTB_ACT_SIGMOID = 4
};
#define NECTB_MAX_LEVELS 24

/* Multiresolution hash encoding (Mueller et al., ACM TOG 41(4) 2022), the
 * encoding the reference builds through tiny-cuda-nn from
 * HashEncoderConfig.get_encoder_config (nect/config.py:86-112).  n_dims is 3
 * (z,y,x) or 4 (z,y,x,t).  Level l has spatial resolution
 * floor(base_resolution * per_level_scale^l) and temporal resolution
 * floor(base_resolution_t * per_level_scale^l) (4D only).  A level is stored
 * densely when its (res+1)^d vertices fit in 2^log2_hashmap_size entries,
 * otherwise it is hashed.  params_f32 layout: level after level, entry after
 * entry, n_features contiguous values per entry; offsets from
 * nectb_hashgrid_layout(). */
typedef struct NectbHashGrid {
  int32_t n_dims;
  int32_t n_levels;
  int32_t n_features;
  int32_t log2_hashmap_size;
  int32_t feature_dtype; /* NECTB_F32 or NECTB_F16 (table storage) */
  double base_resolution;
  double per_level_scale;
  double base_resolution_t;
} NectbHashGrid;

/* Fully connected network without biases (the tiny-cuda-nn FullyFusedMLP the
 * reference configures via MLPNetConfig.get_network_config, nect/config.py:
 * 115-135).  Weights are one fp32 buffer in PyTorch Linear layout
 * ([out][in]): W0 [width x n_input], W1..W_{H-1} [width x width],
 * W_out [1 x width].  compute_dtype NECTB_F32 runs the plain SIMT path;
 * NECTB_BF16 runs the tensor-core path (bf16 operands, fp32 accumulation).
 * The fused model, training and query calls take width 64 and 2 or 3 hidden
 * layers over a grid of 16 levels of 2 or 4 features (n_input 32 or 64) in
 * 3D or 4D, and the reference's default static model (nect/cfg/static/
 * hash_grid.yaml): 6 hidden layers over 19 levels of 4 features (n_input 76)
 * in 3D; hidden activation ReLU on the tensor-core path (LeakyReLU too for
 * the 19-level shape), ReLU, LeakyReLU or none on the SIMT path.  Other
 * shapes return NECTB_ERR_INVALID. */
typedef struct NectbMLP {
  int32_t n_input;
  int32_t n_hidden_layers;
  int32_t width;
  int32_t activation;
  int32_t output_activation;
  int32_t compute_dtype;
} NectbMLP;

/* Per-level layout: resolution, table offset (entries), entries and whether
 * the level is hashed.  Returns the total number of entries. */
int64_t nectb_hashgrid_layout(const NectbHashGrid* grid, int32_t* resolution,
                              int32_t* resolution_t, int64_t* offset,
                              int64_t* entries, int32_t* hashed);
int64_t nectb_mlp_param_count(const NectbMLP* mlp);

/* Encoding of n points x[n*n_dims] (fp32, coordinates in [0,1]) into
 * out[n * n_levels * n_features] fp32.  Replaces the tcnn Encoding forward
 * behind nect/network/networks.py:95-102. */
int nectb_hashgrid_encode(const NectbHashGrid* grid, const void* params,
                          const float* x, int64_t n, float* out, void* stream);

/* Backward of nectb_hashgrid_encode: for n points x[n*n_dims] and the
 * gradient of their encodings dout[n * n_levels * n_features], ADDS
 * sum over points of w_corner * dout into grad (fp32, the table's layout,
 * 16-byte aligned) with fp32 atomics.  Replaces the tcnn Encoding backward
 * behind the reference's composite encodings (nect/network/networks.py:
 * 392-449, QuadCubes). */
int nectb_hashgrid_encode_backward(const NectbHashGrid* grid, const float* x, int64_t n,
                                   const float* dout, float* grad, void* stream);

/* QuadCubes' Composite encoding (nect/network/networks.py:392-449, the
 * reference's default dynamic model): four 3D grids of one configuration
 * (n_dims 3, fp32 tables, 2 or 4 features, the same resolution on every
 * axis) over (z, y, x), (y, x, t), (x, z, t) and (z, y, t) of each point, in
 * the reference's input order (networks.py:438-446).  t is one fp32 value in
 * device memory for every point of the call.
 *
 * nectb_quadcubes_encode writes row i of out (width out_ld, fp32 or bf16 per
 * out_dtype): grid k's n_levels * n_features features at columns
 * [k * L * F, (k + 1) * L * F), then, with identity != 0, the raw inputs
 * (z, y, x, t) (include_identity), then zeros to the end of the row.  The
 * three grids over (a, b, t) are evaluated on their plane at t (the blend of
 * the two time vertices, built in the workspace once per grid and call:
 * fp32, or fp16 when out_dtype is NECTB_BF16), equal to the 3D grid's
 * trilinear interpolation up to fp32 reassociation or that fp16 rounding.
 *
 * nectb_quadcubes_encode_backward adds the table gradients of
 * sum(out[:, :4 * L * F] * dout[:, :4 * L * F]) to grads[0..3] (fp32, the
 * tables' shapes, 16-byte aligned); dout is fp32 or bf16 with rows of width
 * dout_ld; the identity columns carry no gradient (the reference's points do
 * not require one).
 *
 * tables[k] / grads[k] are 4 device pointers in a host array.  out, dout and
 * their rows (ld * element size) are 16-byte aligned.  The workspace (16-byte
 * aligned, nectb_quadcubes_workspace_bytes) holds one plane or one plane
 * gradient at a time; calls on one stream may share it. */
size_t nectb_quadcubes_workspace_bytes(const NectbHashGrid* grid);
int nectb_quadcubes_encode(const NectbHashGrid* grid, const float* const* tables, const float* zyx, int64_t n,
                           const float* t, int identity, void* out, int64_t out_ld, int out_dtype,
                           void* workspace, size_t workspace_bytes, void* stream);
int nectb_quadcubes_encode_backward(const NectbHashGrid* grid, const float* zyx, int64_t n, const float* t,
                                    const void* dout, int64_t dout_ld, int dout_dtype, float* const* grads,
                                    void* workspace, size_t workspace_bytes, void* stream);

/* Diagnostic: per-level corner indices (entry index within the level, int32)
 * and d-linear weights of n points, idx/w[n][n_levels][2^n_dims].  No
 * counterpart in the reference (tiny-cuda-nn keeps them internal); it lets
 * tests check the integer hash arithmetic bit for bit. */
int nectb_hashgrid_corners(const NectbHashGrid* grid, const float* x, int64_t n,
                           int32_t* idx, float* w, void* stream);

/* Model forward sigma = MLP(encode(x)) for n points (queries, export,
 * create_volume).  Replaces NetworkWithInputEncoding forward as called by
 * HashGrid.forward (nect/network/networks.py:59-65) and the export loops
 * (nect/static_export.py:113-138, nect/dynamic_export.py:413-428).  For 4D
 * grids x holds (z,y,x) and t is broadcast (networks.py:85). */
int nectb_model_forward(const NectbHashGrid* grid, const NectbMLP* mlp,
                        const void* grid_params, const float* mlp_params,
                        const float* x, int64_t n, float t, float* sigma,
                        void* stream);

/* Backward of nectb_model_forward: for n points x[n*3] ((z,y,x); t broadcast
 * in 4D) and dsigma[n] = dL/dsigma(x_i), ADDS dL/d(table) into grid_grad
 * (fp32, 16-byte aligned, layout of the fp32 table) and dL/d(weights) into
 * mlp_grad.  Replaces the tiny-cuda-nn backward of direct model calls in the
 * reference's losses on model outputs (the total-variation term on a random
 * 100^3 sub-grid, nect/trainers/base_trainer.py:615-649, nect/utils.py:
 * 64-80).  fp32 SIMT arithmetic for both table precisions. */
int nectb_model_backward(const NectbHashGrid* grid, const NectbMLP* mlp,
                         const void* grid_params, const float* mlp_params,
                         const float* x, int64_t n, float t, const float* dsigma,
                         float* grid_grad, float* mlp_grad, void* stream);

/* nectb_model_forward / nectb_model_backward with the timestep of a 4D grid
 * read from device memory (t: one fp32, broadcast to every point), so a
 * timestep held in a device tensor needs no host synchronisation: the
 * reference broadcasts a 0-d tensor t on the device (nect/network/
 * networks.py:85, 440-444).  Ignored for 3D grids (t must still be valid). */
int nectb_model_forward_t(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                          const float* mlp_params, const float* x, int64_t n, const float* t, float* sigma,
                          void* stream);
int nectb_model_backward_t(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                           const float* mlp_params, const float* x, int64_t n, const float* t,
                           const float* dsigma, float* grid_grad, float* mlp_grad, void* stream);

/* ---- queries -------------------------------------------------------------- */
/* One work item of a query: an nu x nv grid of points
 * x(i, j) = origin + i*du + j*dv (normalised (z,y,x) coordinates, i fast),
 * evaluated at time t and written as sigma*out_scale + out_offset to
 * out[j*out_stride + i].  Slices (axis-aligned or oblique) are one or more
 * items; a volume export is one item per z-slice.  The scale/offset carry the
 * reference's de-normalisation /max_distance_traveled*(max-min)+min
 * (nect/static_export.py:139-140, nect/trainers/base_trainer.py:442-444). */
typedef struct NectbQueryItem {
  float origin[3];
  float du[3];
  float dv[3];
  int32_t nu;
  int32_t nv;
  float t;
  float out_scale;
  float out_offset;
  float* out;
  int64_t out_stride;
  int64_t chunk_begin; /* first 128-point chunk of this item (prefix sum, set by the caller) */
} NectbQueryItem;

/* Evaluates n_items work items (device array) in one persistent launch; the
 * items' chunk_begin must be the exclusive prefix sum of ceil(nu*nv/128).
 * Replaces the per-slice model calls of create_volume / export_volume(s) /
 * export_video (nect/trainers/base_trainer.py:402-450,
 * nect/static_export.py:106-144, nect/dynamic_export.py:297-544), which
 * materialise coordinate grids and call the model one slice at a time.
 * counter: two device uint32: [0] the work cursor (zeroed by every call) and
 * [1] an error word the launch sets to non-zero when a tensor-core wait timed
 * out (its items are then incomplete).  The library never clears [1]: the
 * caller zeroes it once and reads it (stream-ordered) when it wants to know.
 * grid_params must be 16-byte aligned. */
int nectb_query_points(const NectbHashGrid* grid, const NectbMLP* mlp, const void* grid_params,
                       const float* mlp_params, const NectbQueryItem* items, int32_t n_items,
                       int64_t total_chunks, unsigned int* counter, int32_t max_blocks, void* stream);

/* Time slice of a 4D model with an fp16 table: per level, the blend of the
 * two time vertices at t of every entry, w0 * table[e0] + w1 * table[e1]
 * rounded to fp16, in a 3D layout (hashed levels keep the 4D level's hash
 * without its t term; dense levels hold the (res+1)^3 vertices, rounded up
 * to 8 entries).  Queries at that t then gather 8 corners per level instead
 * of 16 (nectb_query_points_slice); the values differ from the 4D
 * interpolation by the fp16 rounding of the blend.  slice_bytes >=
 * nectb_time_slice_bytes(grid), which is 0 for grids without a slice.
 * t in [0, 1].  No reference counterpart (tiny-cuda-nn interpolates the 16
 * corners). */
size_t nectb_time_slice_bytes(const NectbHashGrid* grid);
int nectb_time_slice(const NectbHashGrid* grid, const void* grid_params, float t, void* slice,
                     size_t slice_bytes, void* stream);

/* nectb_query_points on the time slice of a 4D grid (grid describes the 4D
 * model; the items' t is ignored: every point is evaluated at the slice's t). */
int nectb_query_points_slice(const NectbHashGrid* grid, const NectbMLP* mlp, const void* slice,
                             const float* mlp_params, const NectbQueryItem* items, int32_t n_items,
                             int64_t total_chunks, unsigned int* counter, int32_t max_blocks,
                             void* stream);

/* Re-projection of the model: line integrals for every detector pixel of a
 * view at (angle, t), y[p] = sum_s sigma * distances/max_distance_traveled
 * with the training sampler (no jitter, no detector offset), i.e. the
 * reference's training forward (base_trainer.py:520-554) without the loss.
 * The reference has no standalone re-projection query.  workspace:
 * nectb_train_workspace_bytes(geometry, grid, mlp, P) bytes; grid_params
 * 16-byte aligned.
 * max_blocks > 0 caps the persistent grid of either query (a server keeps
 * SMs free for latency-critical launches on higher-priority streams). */
int nectb_query_reproject(const NectbGeometry* geometry, const NectbHashGrid* grid,
                          const NectbMLP* mlp, const void* grid_params, const float* mlp_params,
                          float angle_rad, float t, int32_t num_points_per_ray,
                          float max_ray_distance_per_point, float max_distance_traveled,
                          float* out, void* workspace, size_t workspace_bytes, int32_t max_blocks,
                          void* stream);

/* The detector pixels [pixel_begin, pixel_begin + pixel_count) of the same
 * re-projection (row-major pixel index), written to out[pixel_begin ...]:
 * a server splits a view into pieces of a few milliseconds so that
 * latency-critical launches on higher-priority streams get SMs between them.
 * Values are identical to the whole view's.  workspace:
 * nectb_train_workspace_bytes(geometry, grid, mlp, pixel_count) bytes; a 4D
 * mixed model with nectb_query_reproject_slice_bytes(grid, pixel_count) more
 * bytes gathers 8 corners per level on a time slice at t, built in the
 * workspace by each call, instead of the 16 of the 4D interpolation (the
 * result agrees within fp16 rounding of the blended features).
 * warpgroups_per_sm 1..6: the mixed forward runs one block of that many
 * 128-thread warpgroups per SM, 64 tensor-memory columns each, allocated as
 * a power of two (1, 2, 3-4, 5-6 warpgroups take 64, 128, 256, 512 of an
 * SM's 512 columns; up to 4 leave room for query blocks on other streams);
 * 0 = max_blocks' rule.
 * No reference counterpart. */
int nectb_query_reproject_range(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                const NectbMLP* mlp, const void* grid_params, const float* mlp_params,
                                float angle_rad, float t, int32_t num_points_per_ray,
                                float max_ray_distance_per_point, float max_distance_traveled,
                                float* out, int32_t pixel_begin, int32_t pixel_count, void* workspace,
                                size_t workspace_bytes, int32_t max_blocks, int32_t warpgroups_per_sm,
                                void* stream);

/* Extra workspace bytes that let nectb_query_reproject_range run a 4D mixed
 * model on a time slice (0 for other models). */
size_t nectb_query_reproject_slice_bytes(const NectbHashGrid* grid, const NectbMLP* mlp,
                                         int32_t pixel_count);

/* ---- fused training step ------------------------------------------------ */
/* One batch of rays from one projection.  Fuses Projector.__call__
 * (nect/sampling/projector.py:102-131), the zero-point mask and chunked
 * model calls (nect/trainers/base_trainer.py:523-551), the line integral
 * (:552-554), the loss (nect/config.py:481-497) and its backward
 * (base_trainer.py:650): positions and encodings never reach HBM.
 * measured[num_rays] are the projection values proj[perm[start:start+R]]
 * (already gathered by the caller or gathered here when measured_full is
 * given, see nectb_train_step).  Outputs y_pred[num_rays], loss (mean over
 * rays), and gradients ADDED into grid_grad (fp32, same layout as the fp32
 * table) and mlp_grad (fp32).  loss_type: 1 = L1, 2 = L2.  scale =
 * distances/max_distance_traveled factor is computed in-kernel. */
typedef struct NectbTrainBatch {
  const int64_t* random_ray_index;
  int64_t random_ray_index_len;
  int64_t starting_ray_index;
  int32_t num_rays;
  int32_t num_points_per_ray;
  float angle_rad;
  float t;                          /* timestep in [0,1] (4D grids) */
  float max_ray_distance_per_point;
  int32_t uniform_ray_spacing;
  float max_distance_traveled;
  const float* jitter;              /* [num_rays]   */
  const float* detector_offset;     /* [num_rays*2] */
  const float* projection;          /* full flattened projection [P] */
  int32_t loss_type;
  float loss_scale;                 /* multiplies dL/dy (1 = plain mean) */
} NectbTrainBatch;

size_t nectb_train_workspace_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                   const NectbMLP* mlp, int32_t num_rays);

/* Recommended staging bytes for the mixed path's two-pass backward, to add to
 * nectb_train_workspace_bytes(): the rays with samples are listed in
 * scheduling order (detector pixels, or batch positions when the batch
 * repeats a pixel) and the backward runs in rounds of equal ray counts
 * (NectbTuning::staged_rounds, 4 by default);
 * each round's tensor-core pass writes dL/d(encoding) of its samples (fp32,
 * num_points_per_ray * n_levels * n_features per ray) and scatter passes over
 * level groups apply it to grid_grad with the gradient slice of each group
 * resident in L2.  The rounds' part is capped at 16 GiB (plus the ray list).
 * It also includes an encoding store: the forward writes each sample's bf16
 * MLP input row (n_levels * n_features * 2 bytes) there and the backward
 * reads it back instead of gathering the tables a second time (identical
 * values); the store has a row for every sample slot (num_rays *
 * num_points_per_ray), capped at 80 GiB, and rays whose rows do not fit
 * gather again.  A smaller buffer gets fewer store rows, then no store, then
 * more rounds; when it would take more than 64 rounds the single-pass
 * backward (scatter inside the tensor-core kernel) runs instead.  The split
 * between store and rounds follows the buffer size and staged_rounds, so a
 * split step's two halves take the same workspace size with the tuning
 * unchanged between them.  Returns 0 for the plain fp32 path, which does
 * not stage.  No reference counterpart. */
size_t nectb_train_staging_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                 const NectbMLP* mlp, int32_t num_rays, int32_t num_points_per_ray);

/* Device address of the error word inside a training (or re-projection)
 * workspace of num_rays rays (num_rays = detector pixels for a
 * re-projection); workspace NULL gives the word of the static scratch of
 * nectb_train_step_static on the current device (NULL, with
 * NECTB_ERR_TOO_LARGE as the last error, for a batch that scratch cannot
 * hold).  Every step clears the word
 * and sets it to non-zero when a tensor-core wait of that step timed out
 * (results of the step are then incomplete and the call's stream stays
 * usable).  Read it stream-ordered after the step, e.g. with cudaMemcpyAsync.
 * Returns NULL on invalid arguments.  No reference counterpart (the reference
 * reports only CUDA errors, ct_sampling.cu:639-644). */
const unsigned int* nectb_train_error_word(const NectbGeometry* geometry, int32_t num_rays,
                                           const void* workspace);

/* Diagnostic of the fused path's sampling: the rays a training step (or its
 * forward half) prepared in a workspace of num_rays rays, read back after
 * it.  counts[num_rays] int32: the samples the fused kernels evaluate per
 * ray, the reference sampler's written samples (ct_sampling.cu:475-576);
 * scale[num_rays] fp32: distances[r] / max_distance_traveled, the factor of
 * the line integral (base_trainer.py:552-554); points[num_rays *
 * num_points_per_ray * 3] fp32 (z,y,x): the positions the fused kernels
 * regenerate for samples 0..S-1, after the Projector clamp
 * (projector.py:127), 0 beyond the count, i.e. the reference's sample()
 * output after clamp_(0, 1).  Any output may be NULL.  Stream-ordered.  No
 * reference counterpart: the reference's fused equivalent does not exist,
 * its sampler writes these to HBM. */
int nectb_train_rays(const NectbGeometry* geometry, int32_t num_rays, int32_t num_points_per_ray,
                     const void* workspace, int32_t* counts, float* scale, float* points, void* stream);

/* Fused forward+backward.  grid_params is the table in grid->feature_dtype
 * (fp32 or fp16); mlp_params fp32; grid_params and grid_grad 16-byte
 * aligned (paired 16-byte reductions).  Gradients are accumulated (+=) into
 * grid_grad (fp32, nectb_hashgrid_layout total * n_features) and mlp_grad
 * (fp32, nectb_mlp_param_count).  y_pred[num_rays] and loss[1] are written.
 * workspace: at least nectb_train_workspace_bytes() bytes of device memory;
 * bytes beyond that are staging for the mixed path's two-pass backward
 * (nectb_train_staging_bytes). */
int nectb_train_step(const NectbGeometry* geometry, const NectbHashGrid* grid,
                     const NectbMLP* mlp, const void* grid_params,
                     const float* mlp_params, const NectbTrainBatch* batch,
                     float* grid_grad, float* mlp_grad, float* y_pred,
                     float* loss, void* workspace, size_t workspace_bytes,
                     void* stream);

/* The step in two halves, for losses of y_pred that the caller computes
 * itself (the reference composes y_pred, then loss_fn(y_pred, y), optional
 * Poisson noise and S3IM, base_trainer.py:552-566; continuous-scan training
 * averages y_pred over several sub-angles, continous_scanning_trainer.py:
 * 85-140).  nectb_train_forward prepares the rays and writes y_pred[num_rays]
 * (loss_type and loss_scale are ignored); nectb_train_backward then takes
 * dloss_dy[num_rays] = dL/dy_pred and ADDS the gradients into grid_grad and
 * mlp_grad.  Both get the same batch and the same workspace, which must not be
 * used by another step in between; positions and encodings are regenerated in
 * the backward, as in nectb_train_step. */
int nectb_train_forward(const NectbGeometry* geometry, const NectbHashGrid* grid,
                        const NectbMLP* mlp, const void* grid_params,
                        const float* mlp_params, const NectbTrainBatch* batch,
                        float* y_pred, void* workspace, size_t workspace_bytes,
                        void* stream);
int nectb_train_backward(const NectbGeometry* geometry, const NectbHashGrid* grid,
                         const NectbMLP* mlp, const void* grid_params,
                         const float* mlp_params, const NectbTrainBatch* batch,
                         const float* dloss_dy, float* grid_grad, float* mlp_grad,
                         void* workspace, size_t workspace_bytes, void* stream);

/* Continuous-scan training step (nect/trainers/continous_scanning_trainer.py:
 * 85-140): the detector integrates while the object turns, so each pixel's
 * prediction is the mean over sub_angles (1..32) sub-angles of its line
 * integral, y_pred[r] = sum_j (sum_s sigma_jrs * distances_jr /
 * max_distance_traveled) / sub_angles, with every sub-angle ray of the pixel
 * at the batch's t.  All sub-angle rays of the batch (sub_angles *
 * num_rays) run through ONE launch of each fused kernel instead of one
 * forward per sub-angle.  sub_angles_rad: host array of the sub angles
 * (batch->angle_rad is ignored); batch->jitter holds sub_angles * num_rays
 * and batch->detector_offset sub_angles * num_rays * 2 draws, sub-angle-major
 * (the reference draws them per sub-angle call of sample(), in that order).
 * y_pred[num_rays]; loss = mean over the num_rays pixels; gradients are
 * ADDED.  The forward/backward halves take dL/dy_pred per pixel.  Workspace:
 * nectb_train_scan_workspace_bytes() plus, for the mixed path's two-pass
 * backward, nectb_train_scan_staging_bytes(); its error word is
 * nectb_train_scan_error_word().  No other reference counterpart. */
size_t nectb_train_scan_workspace_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                        const NectbMLP* mlp, int32_t num_rays, int32_t sub_angles);
size_t nectb_train_scan_staging_bytes(const NectbGeometry* geometry, const NectbHashGrid* grid,
                                      const NectbMLP* mlp, int32_t num_rays, int32_t num_points_per_ray,
                                      int32_t sub_angles);
int nectb_train_scan_step(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                          const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                          const float* sub_angles_rad, int32_t sub_angles, float* grid_grad, float* mlp_grad,
                          float* y_pred, float* loss, void* workspace, size_t workspace_bytes, void* stream);
int nectb_train_scan_forward(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                             const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                             const float* sub_angles_rad, int32_t sub_angles, float* y_pred, void* workspace,
                             size_t workspace_bytes, void* stream);
int nectb_train_scan_backward(const NectbGeometry* geometry, const NectbHashGrid* grid, const NectbMLP* mlp,
                              const void* grid_params, const float* mlp_params, const NectbTrainBatch* batch,
                              const float* sub_angles_rad, int32_t sub_angles, const float* dloss_dy,
                              float* grid_grad, float* mlp_grad, void* workspace, size_t workspace_bytes,
                              void* stream);
const unsigned int* nectb_train_scan_error_word(const NectbGeometry* geometry, int32_t num_rays,
                                                int32_t sub_angles, const void* workspace);

/* nectb_train_step without a caller workspace, for callers that cannot
 * allocate device memory (a runtime that binds this library through its C ABI
 * and has no CUDA allocator, or a loop that must never call cudaMalloc, which
 * synchronises the device and can fail mid-run).  No counterpart in the
 * reference.  Scratch is a library-owned __device__ array of
 * nectb_train_static_scratch_bytes() (20 MiB + 4 KiB) that every GPU loading
 * the library reserves until exit; batches needing more (above 262,144 rays
 * on a 1024x1024 detector) fail with NECTB_ERR_TOO_LARGE.  Every call (its
 * device current) looks up the array's address, which allocates nothing; the
 * first call on a device loads the library's module there, so make it before
 * any stream capture.  Calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller.  Allocates nothing. */
int nectb_train_step_static(const NectbGeometry* geometry, const NectbHashGrid* grid,
                            const NectbMLP* mlp, const void* grid_params,
                            const float* mlp_params, const NectbTrainBatch* batch,
                            float* grid_grad, float* mlp_grad, float* y_pred,
                            float* loss, void* stream);
size_t nectb_train_static_scratch_bytes(void);

/* Adam (torch.optim.Adam semantics, as configured in nect/config.py:400-414)
 * over n fp32 parameters with fp32 moments; step is the 1-based step count.
 * The hyper-parameters are doubles, as torch holds them: 1 - beta1,
 * 1 - beta2, lr / (1 - beta1^step) and sqrt(1 - beta2^step) are formed in
 * double before the fp32 update, in torch's order of operations.  When
 * param_half is non-NULL the updated parameter is also written there as
 * fp16 (the mixed path's table copy).  grad is zeroed after use when
 * zero_grad != 0 (optim.zero_grad, base_trainer.py:518). */
int nectb_adam_step(float* param, float* grad, float* exp_avg, float* exp_avg_sq,
                    int64_t n, double lr, double beta1, double beta2, double eps,
                    double weight_decay, int32_t step, void* param_half,
                    int32_t zero_grad, void* stream);

/* Per-kernel timing of the library's own launches with CUDA events recorded
 * on the launch stream around each kernel (off by default).  Slots:
 * 0 ray preparation, 1 forward, 2 backward, 3 Adam, 4 sampling, 5 model
 * forward and queries, 6 staged gradient scatter, 7 ray ordering of the
 * staged backward (three launches timed as one), 8 time slice of a 4D grid
 * and the spread of its gradient.  nectb_profile_collect waits for the
 * recorded events, adds their durations and returns per slot the launch
 * count and total milliseconds.  No counterpart in the reference, which has
 * no profiler. */
#define NECTB_PROFILE_SLOTS 9
int nectb_profile_enable(int32_t enable);
int nectb_profile_collect(int32_t* launches, double* total_ms);

/* Self-test of the bounded waits the tensor-core kernels use: one block waits
 * on an mbarrier that nothing arrives at, polling at most max_tries times,
 * then writes *error_word = 1 if the wait gave up (0 if it completed).  It
 * lets a test check, on a GPU and without any fault, that a wait that runs
 * out ends the kernel with a status the host reads and leaves the context
 * usable.  No reference counterpart. */
int nectb_selftest_bounded_wait(unsigned int* error_word, uint32_t max_tries, void* stream);

/* Launch shapes and scheduling of the mixed training path, process-wide:
 * warpgroups per SM of the forward (1..6), blocks per SM of the tensor-core
 * backward (1..3; the three-layer model's kernel takes at most 2),
 * of the gradient scatter (0 = as many as fit), the rounds the recommended
 * staging is sized for (nectb_train_staging_bytes, 1..64), the largest fp32
 * gradient slice one scatter pass covers, and the samples-per-cell
 * thresholds above which runs of samples along a ray are merged before their
 * reductions (3D and 4D grids), and time_slice: 1 lets a mixed 4D training
 * step with staging interpolate the fp16 table at the batch's t once (a 3D
 * slice per level, fp16) and run the 3D kernels on it, the gradient being
 * spread back to the two time vertices afterwards; the slice's fp16 rounding
 * lies below the bf16 rounding of the MLP input.  The other settings change
 * results by fp32 reassociation only; the Python autotuner
 * (nect_b200.autotune) picks them per workload.  encoding_store: 1 lets the
 * mixed forward keep each sample's bf16 MLP input row in the staging region
 * for the backward to read back; 0 recomputes the encodings in the backward
 * from the tables (positions are always regenerated), so the staging holds
 * only the ray order and the staged gradients (identical results: the
 * stored rows are the bits the gather produces).  nectb_train_staging_bytes
 * follows it.  nectb_set_tuning validates and applies to steps issued after
 * it returns; defaults: 6, 3, 0, 4, 48 MiB, 1.0, 3.0, 1, 1.  No reference
 * counterpart. */
typedef struct NectbTuning {
  int32_t forward_blocks_per_sm;
  int32_t backward_blocks_per_sm;
  int32_t scatter_blocks_per_sm;
  int32_t staged_rounds;
  int64_t scatter_group_bytes;
  float run_threshold_3d;
  float run_threshold_4d;
  int32_t time_slice;
  int32_t encoding_store;
} NectbTuning;
int nectb_get_tuning(NectbTuning* tuning);
int nectb_set_tuning(const NectbTuning* tuning);

/* Roofline probes (no reference counterpart): the measured roofs that the
 * encoding's corner gathers and the gradient scatter's reductions are
 * reported against.  nectb_probe_gather loads entry_bytes (4, 8, 16, or 32 =
 * one whole L2 sector) from entries of buf[n_entries * entry_bytes];
 * nectb_probe_reduce (4, 8 or 16 bytes) adds fp32 values with one
 * entry_bytes-wide reduction into entries of buf.  mode 0: every lane takes
 * its own random entry (hashed corners); mode 1: the 32 lanes of a warp take
 * 32 consecutive entries at a random 32-entry boundary (whole lines: the
 * memory system's byte bandwidth).  Both run about n_ops accesses, exactly
 * nectb_probe_ops(n_ops), in one launch of 64 warps per SM on the stream; the
 * caller times them.  A buffer below the L2 size gives the L2 roof, a larger
 * one the HBM random-access roof.  sink: one device uint32 the gather probe
 * may write. */
int nectb_probe_gather(const void* buf, int64_t n_entries, int32_t entry_bytes, int32_t mode, int64_t n_ops,
                       unsigned int* sink, void* stream);
int nectb_probe_reduce(float* buf, int64_t n_entries, int32_t entry_bytes, int32_t mode, int64_t n_ops,
                       void* stream);
int64_t nectb_probe_ops(int64_t n_ops);

/* Version string and last error message of the calling thread. */
const char* nectb_version(void);
const char* nectb_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* NECTB_H_ */
