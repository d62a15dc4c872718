/* spectral.h -- C ABI of the B200 spectral path-tracing library (libspectral.so).
 *
 * Drop-in for the Taichi kernels and module-global fields of
 * Xyzonox/taichi-spectral-render main.py.  Every entry point names the
 * reference code it replaces.  Conventions:
 *   - every call returns ts_status; on failure ts_last_error() describes it;
 *   - device pointers are CUDA device addresses on the context's device;
 *     "stream" is a cudaStream_t (NULL = the legacy default stream); calls are
 *     stream-ordered and a context must not be used from two threads at once;
 *   - scene arrays are caller-owned host memory, copied during the call;
 *   - pixel (i, j): i is the column (0..width-1), j the row counted from the
 *     bottom, as the reference indexes pixels_geometry[i, j] (main.py:1505).
 */
#ifndef TS_SPECTRAL_H
#define TS_SPECTRAL_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ts_ctx ts_ctx;

typedef enum {
  TS_OK = 0,
  TS_ERR_INVALID_ARG = 1,
  TS_ERR_CUDA = 2,
  TS_ERR_OUT_OF_MEMORY = 3,
  TS_ERR_CAPACITY = 4,      /* a queue or table bound was exceeded */
  TS_ERR_DEVICE_FAULT = 5,  /* a kernel reported an error bit (stack overflow, iteration cap) */
  TS_ERR_NO_SCENE = 6
} ts_status;

/* Render kernels */
enum { TS_KERNEL_MEGA = 0, TS_KERNEL_WAVEFRONT = 1 };
/* Traversal loop of the two-child BVH layout (ts_config.traversal) */
enum { TS_TRAVERSAL_DEFAULT = 0, TS_TRAVERSAL_SPECULATIVE = 1 };
/* Traversal modes of ts_trace_batch */
enum { TS_TRACE_FAST = 0, TS_TRACE_REFERENCE_ORDER = 1 };
/* Film buffers */
enum { TS_FILM_BLOCK = 0, TS_FILM_MEAN = 1, TS_FILM_M2 = 2 };

/* Render constants of main.py:11-35 as runtime values. */
typedef struct {
  int32_t width, height;         /* RENDER_WIDTH, RENDER_HEIGHT */
  int32_t bands;                 /* SPECTRAL_BANDS (1..64) */
  float lambda_min_nm, lambda_max_nm; /* WAVELENGTH_MIN, WAVELENGTH_MAX */
  int32_t max_path_length;       /* MAX_PATH_LENGTH */
  int32_t scatter_bounces;       /* SCATTER_BOUNCES (shadow segments) */
  float epsilon, escape;         /* EPSILON, ESCAPE */
  float aspect_ratio;            /* ASPECT_RATIO */
  float fov_scale;               /* 1.0 = the reference's fixed half-FOV atan(1/2); s gives atan(s/2) */
  uint32_t seed;                 /* Philox key word 0 (word 1 is the pass index) */
  uint32_t scene_id;             /* Philox counter word 2 (distinguishes scenes of a batch) */
  int32_t device;                /* CUDA device ordinal */
  int32_t kernel;                /* TS_KERNEL_MEGA or TS_KERNEL_WAVEFRONT */
  int32_t block_size;            /* threads per block of the render kernels, 32..256 (0 = 128) */
  int32_t blocks_per_sm;         /* persistent grid = SMs * blocks_per_sm (0 = default) */
  int32_t sort_keys;             /* wavefront queue sorting, bit mask: 1 shading queue by material,
                                    2 extension rays by direction octant, 4 shadow rays by light (0 = off) */
  int32_t trace_budget;          /* wavefront: traversal steps between refills of idle lanes (0 = 32) */
  int32_t traversal;             /* TS_TRAVERSAL_DEFAULT or TS_TRAVERSAL_SPECULATIVE (two-child nodes) */
  int32_t occupancy;             /* megakernel register budget: 0 = 5 resident blocks of 128 per SM (96 registers),
                                    8 = 8 blocks (64 registers, spills; more latency hiding on large frames) */
  int32_t queue_capacity;        /* wavefront path slots (0 = one per pixel; at most 2^25).  With sort_keys == 0,
                                    ts_render_passes, and ts_render_pass when queue_capacity > 0, run the
                                    regenerating loop: a slot whose path has ended starts the next pixel (of
                                    the next pass of a bundle) at once, so several passes can be in flight.
                                    With sort_keys != 0 a pass is rendered depth-synchronously in chunks of at
                                    most queue_capacity pixels. */
  int32_t loop_host;             /* regenerating loop: 0 = the iterations run as a CUDA-graph while-loop;
                                    1 = the host launches them, reading the loop's continue flag after each
                                    (one stream synchronisation per iteration: for profilers that do not
                                    descend into conditional graph nodes).  Results are identical. */
} ts_config;

/* Scene in the reference's data model (setup_scene, main.py:509-631). Triangles
 * are given in ORIGINAL order; the library reorders them into BVH order. */
typedef struct {
  int32_t num_tris;
  const float *v0, *v1, *v2;        /* [T][3] vertices */
  const float *n0, *n1, *n2;        /* [T][3] vertex normals (the face normal where the mesh has none) */
  const float *normal;              /* [T][3] unit geometric normal, as main.py:525-534 computes it */
  const float *area;                /* [T] triangle area */
  const int32_t *mat_id;            /* [T] */
  int32_t num_materials;
  const float *mat_f32;             /* [M][6][B]: n, k, roughness, scattering, emission, anisotropy */
  const int32_t *mat_i32;           /* [M][2][B]: is_true_volume, surface_emission */
  const int32_t *mat_eem;           /* [M]: EEM id (0 = none) */
  int32_t num_eems;                 /* rows of eem, including the unused id 0 */
  const float *eem;                 /* [E][B][B], row = excitation band (may be NULL if num_eems == 0) */
  const float *cmf;                 /* [B][3] colour-matching functions at the band centres */
  /* BVH: bvh_num_nodes == 0 builds one (binned SAH); otherwise the tree is
   * adopted as given in the reference layout (main.py:267-275, e.g. the
   * output of the reference's build_bvh), with tri_perm[slot] = original index. */
  int32_t bvh_num_nodes;
  const float *node_min, *node_max; /* [N][3] */
  const int32_t *node_left, *node_right, *node_num_tris, *node_tri_start, *tri_perm;
  /* binned-SAH parameters (0 = defaults) */
  int32_t bvh_bins, bvh_leaf_max;
  float bvh_cost_trav, bvh_cost_tri;
  int32_t bvh_width;                /* device node width 2, 4 or 8 (0 = library default) */
  int32_t bvh_quantized;            /* 4- and 8-wide nodes: nonzero stores each child box as 8-bit offsets from the
                                       node's origin, rounded outwards (64 / 96 B per node instead of 128 / 256 B;
                                       the boxes only grow, so closest hits are unchanged) */
} ts_scene_desc;

typedef struct {
  int32_t num_tris, num_nodes, num_ref_nodes, max_depth, leaves;
  double sah_cost;
  int32_t max_lights;
  size_t device_bytes;  /* device memory held by the context */
  int32_t node_width;   /* node width of the uploaded device BVH */
  int32_t node_quantized; /* its child boxes are quantized (ts_scene_desc.bvh_quantized) */
} ts_scene_info;

/* ---- context (replaces ti.init + the module-global fields, main.py:9, 361-394) */
ts_status ts_create(const ts_config *cfg, ts_ctx **out);
ts_status ts_destroy(ts_ctx *ctx);
/* Change the launch settings of a context -- kernel, traversal, block_size,
 * blocks_per_sm, sort_keys, trace_budget, occupancy, queue_capacity, loop_host of *cfg; every other field is
 * ignored -- without re-uploading the scene (the autotuner's knob).  Paths and
 * images do not depend on these settings. */
ts_status ts_set_launch_config(ts_ctx *ctx, const ts_config *cfg);
const char *ts_last_error(const ts_ctx *ctx); /* ctx may be NULL: last error of this thread */
const char *ts_version(void);

/* ---- scene (setup_scene + build_bvh + get_scene_dimensions, main.py:398-631) */
ts_status ts_upload_scene(ts_ctx *ctx, const ts_scene_desc *scene);
ts_status ts_scene_info_get(const ts_ctx *ctx, ts_scene_info *info);

/* A view of another context's scene (new; the reference renders one camera of
 * one scene): a context with its own config (resolution, depth, seed, scene id,
 * launch settings), camera and film that renders the owner's uploaded scene
 * without uploading or copying it.  Bands and wavelength range must equal the
 * owner's.  The owner must outlive its views; the material tables are shared
 * (ts_update_materials through either updates both); ts_upload_scene on a
 * view gives it a scene of its own.  Views batch like any context. */
ts_status ts_create_view(const ts_ctx *owner, const ts_config *cfg, ts_ctx **out);
/* slot -> original triangle index, [num_tris] host array */
ts_status ts_get_tri_perm(const ts_ctx *ctx, int32_t *perm_out);

/* Host-only BVH build (replaces build_bvh, main.py:437-507): the binned-SAH
 * tree ts_upload_scene would build, returned in the reference layout.
 * Output arrays hold max_nodes entries (2*num_tris-1 always suffices);
 * tri_perm[slot] = original triangle index.  Needs no GPU. */
ts_status ts_build_bvh_host(int32_t num_tris, const float *v0, const float *v1, const float *v2, int32_t bins,
                            int32_t leaf_max, float cost_trav, float cost_tri, int32_t max_nodes, float *node_min,
                            float *node_max, int32_t *node_left, int32_t *node_right, int32_t *node_num_tris,
                            int32_t *node_tri_start, int32_t *tri_perm, int32_t *num_nodes_out);

/* ---- camera (update_camera, main.py:633-640) */
ts_status ts_set_camera(ts_ctx *ctx, const float origin[3], const float lookat[3], const float up[3]);

/* ---- render (cast_rays(current_sample_in_block, block_index), main.py:1502-1590).
 * pass_idx selects the random stream (Philox key word 1); band is the pass's
 * wavelength index (current_sample_in_block).  Deposits into TS_FILM_BLOCK. */
ts_status ts_render_pass(ts_ctx *ctx, uint32_t pass_idx, int32_t band, void *stream);

/* num_passes consecutive passes in one launch (a wavelength bundle): pass
 * first_pass + i renders band (first_band + i) mod B, 1 <= num_passes <= B so
 * that every pass owns its own film plane; the same paths and deposits as
 * num_passes ts_render_pass calls (film sums equal up to the order of FP64
 * additions where volume fluorescence moves deposits between bands).  Small frames fill the GPU this way.  The
 * wavefront kernel runs it as the regenerating loop (sort_keys == 0: one init kernel, then a CUDA graph
 * whose while-loop iterates trace -> shade until the queues are empty), or one depth-synchronous launch
 * sequence per pass (sort_keys != 0). */
ts_status ts_render_passes(ts_ctx *ctx, uint32_t first_pass, int32_t num_passes, int32_t first_band, void *stream);

/* Loop iterations of the last regenerating wavefront launch (each one trace,
 * one shade and one control kernel); synchronises the stream.  0 before any. */
ts_status ts_wave_loop_iterations(ts_ctx *ctx, void *stream, int32_t *iterations);

/* Bound on the iterations of one regenerating-loop launch (new; the reference
 * has no device-side loop).  0 (the default) = the automatic bound, which no
 * launch reaches unless its queues are corrupt: every slot starts a new work
 * item at least once per max_path_length iterations while items are left.  A
 * smaller positive limit applies when tighter.  A launch that reaches the
 * bound stops on the device (its remaining paths are dropped) and sets the
 * iteration-cap bit that ts_check_device reports as TS_ERR_DEVICE_FAULT; the
 * next launch starts clean.  For failure-handling tests and watchdogs. */
ts_status ts_set_loop_iteration_limit(ts_ctx *ctx, int32_t limit);

/* The same pass rendered by the plain megakernel with work counters (used to
 * derive algorithmic bytes per path).  work[0..6] = paths, path vertices,
 * traversals, BVH node visits, triangle tests, hits resolved, film deposits;
 * work[7] unused.  Deposits into TS_FILM_BLOCK like ts_render_pass; the
 * stream is synchronised. */
ts_status ts_render_pass_counted(ts_ctx *ctx, uint32_t pass_idx, int32_t band, void *stream, uint64_t work[8]);

/* Allocation-free render of one tile (no counterpart in the reference, whose
 * Taichi runtime allocates everything up front).  For callers that cannot
 * call cudaMalloc while they render -- an application whose device-memory
 * budget is fixed after start-up, or a render loop inside another framework
 * that owns the allocator -- where ts_render_pass's wavefront kernel would
 * allocate its path-state buffers on first use.  Renders pass pass_idx / band
 * for the pixels [x0, x0+tile_w) x [y0, y0+tile_h) of the context's scene and
 * camera, with the same random streams as ts_render_pass, ADDING deposits into
 * film_dev: a caller-owned [B][H][W] float64 device buffer of the frame.
 * At most 65536 pixels per call (TS_ERR_CAPACITY beyond).  Its scratch is a
 * static device array of about 8.4 MB that every GPU using it keeps until
 * exit.  The CUDA runtime loads it lazily: the first call on a device (or an
 * earlier wavefront launch of this library there) reserves the array and
 * looks its address up, so a host with a fixed memory budget makes that first
 * call during start-up, before any stream capture.  The address is looked up
 * again in a new context (after a device reset).  All calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller. */
ts_status ts_render_tile_noalloc(ts_ctx *ctx, uint32_t pass_idx, int32_t band, int32_t x0, int32_t y0,
                                 int32_t tile_w, int32_t tile_h, double *film_dev, void *stream);

/* ---- film (average_and_reset_block, clear_pixel_space, main.py:1592-1607, 1661-1674) */
ts_status ts_accumulate_block(ts_ctx *ctx, int32_t num_blocks_completed, void *stream);
ts_status ts_reset(ts_ctx *ctx, void *stream);
/* device pointer + element count of a film buffer ([B][H][W] float64) */
ts_status ts_film_buffer(ts_ctx *ctx, int32_t which, double **dev_ptr, size_t *count);
/* copy a film buffer to host memory (synchronises the stream) */
ts_status ts_film_download(ts_ctx *ctx, int32_t which, double *host, void *stream);

/* ---- resolve (color_rays, main.py:1609-1629).  scale multiplies the CMF dot
 * product: WAVELENGTH_STEP / normalization_factor in the reference.
 * xyz_dev: [H][W][3] float32 device buffer. */
ts_status ts_resolve_xyz(ts_ctx *ctx, double scale, float *xyz_dev, void *stream);
/* same, into a host buffer (device scratch, copy back, stream synchronised) */
ts_status ts_resolve_xyz_host(ts_ctx *ctx, double scale, float *xyz_host, void *stream);
/* full color_rays: upscale to img_w x img_h, XYZ->RGB (row-major 3x3), Reinhard, gamma. */
ts_status ts_resolve_rgb(ts_ctx *ctx, double scale, const float xyz_to_rgb[9], float exposure, float gamma,
                         int32_t img_w, int32_t img_h, float *rgb_dev, void *stream);

/* ---- geometry (trace, main.py:831-864; visualize_normals, main.py:1631-1659) */
/* rays_dev: [n][6] (origin, direction); outputs [n] device arrays, tri = original
 * triangle index or -1, t = 1e9 on a miss; u/v may be NULL. */
ts_status ts_trace_batch(ts_ctx *ctx, const float *rays_dev, int32_t n, int32_t mode, int32_t *tri_dev,
                         float *t_dev, float *u_dev, float *v_dev, void *stream);
/* normals_dev: [H][W][3] float32 */
ts_status ts_render_normals(ts_ctx *ctx, float *normals_dev, void *stream);

/* ---- differentiation (new; the reference renders forward only).
 * Parameters are the material table [M][6][B] of ts_scene_desc.mat_f32
 * (main.py:545-561) followed by the EEM table [E][B][B]; gradients exist for
 * every entry except the refractive index (property 0), which bends rays.
 * Counts: M*6*B material entries, E*B*B EEM entries. */
ts_status ts_param_count(const ts_ctx *ctx, int64_t *num_material_params, int64_t *num_eem_params);

/* Replace the material and/or EEM tables (device arrays in the ts_scene_desc
 * layout; either may be NULL) without touching geometry, BVH or lights: the
 * parameter update of an optimiser.  The integer flags (is_true_volume,
 * surface_emission) and EEM ids stay as uploaded.  Stream-ordered. */
ts_status ts_update_materials(ts_ctx *ctx, const float *mat_f32_dev, const float *eem_dev, void *stream);

/* Path records (new): arm recording for passes first_pass .. first_pass +
 * num_passes - 1 (num_passes = 0 disarms; allocates num_passes * W * H floats
 * here, not while rendering).  Renders of armed passes (ts_render_pass, and
 * ts_render_passes whose passes all fall in the range) run the megakernel and
 * write each path's total deposit.  A later ts_adjoint_passes over recorded
 * passes at the same bands then skips its weight replay for every path that
 * stayed in its band (the weight is the adjoint film at the path's cell times
 * the recorded total); the gradients are the same.  Uploading a scene, moving
 * the camera or updating the materials marks the records stale. */
ts_status ts_record_paths(ts_ctx *ctx, uint32_t first_pass, int32_t num_passes);

/* Path-replay adjoint of ts_render_pass(pass_idx, band): re-runs each path of
 * that pass from its random stream and ADDS into grad_dev ([M*6*B + E*B*B]
 * float64, device) the derivative of sum over the pass's film deposits of
 * adj[band'][j][i] * deposit, where adj_dev is a [B][H][W] float64 device
 * array (dLoss/d film cell).  Sampling decisions that depend on a parameter
 * contribute their score terms, so the result is the gradient of the expected
 * pass.  scatter_bounces must be <= 16. */
ts_status ts_adjoint_pass(ts_ctx *ctx, uint32_t pass_idx, int32_t band, const double *adj_dev, double *grad_dev,
                          void *stream);
/* The adjoint of num_passes consecutive passes (pass first_pass + i at band
 * (first_band + i) mod B) in one launch; any num_passes >= 1. */
ts_status ts_adjoint_passes(ts_ctx *ctx, uint32_t first_pass, int32_t num_passes, int32_t first_band,
                            const double *adj_dev, double *grad_dev, void *stream);

/* ---- batched rendering (new; the reference renders one scene at a time).
 * Many scenes -- each a context with its own scene, camera, resolution, depth
 * and film -- rendered by one persistent kernel per step.  A step renders one
 * whole spectral block of every active scene (band b at pass first_pass +
 * B*k + b in its k-th step) and then does its average_and_reset_block; the
 * paths are exactly those of ts_render_pass on each context (film sums equal
 * up to the order of FP64 additions where fluorescence moves deposits between
 * bands).  The batch
 * snapshots the contexts' scenes, cameras and films at creation: contexts must
 * outlive the batch and keep their scene uploaded.  All scenes must live on
 * one device and share the BVH width and traversal variant.  Internally the
 * work pool puts the deepest scenes first; arguments stay in the caller's
 * scene order. */
typedef struct ts_batch ts_batch;
typedef struct {
  int32_t block_size;     /* megakernel: threads per block, 32..128 (0 = 128) */
  int32_t blocks_per_sm;  /* megakernel: persistent grid = SMs * blocks_per_sm (0 = 5) */
  int32_t use_graph;      /* 1: capture a step as one CUDA graph at the first step, replay it after */
  int32_t occupancy;      /* megakernel: 0 = 5 resident blocks per SM (96 registers), 8 = 8 blocks (64 registers) */
  int32_t kernel;         /* TS_KERNEL_MEGA: one persistent megakernel per step; TS_KERNEL_WAVEFRONT: one
                             regenerating wavefront loop over every active scene's block per step (init kernel,
                             then a while-loop of trace -> shade over all scenes' paths), the whole step one
                             CUDA graph with use_graph */
  int32_t queue_capacity; /* wavefront: path slots shared by all scenes (0 = min(paths per step, 2^24); at most
                             2^25; 160 B of device memory per slot) */
  int32_t trace_budget;   /* wavefront: traversal steps between refills of idle lanes (0 = 16) */
} ts_batch_config;

ts_status ts_batch_create(const ts_batch_config *cfg, ts_ctx *const *ctxs, int32_t num_scenes, ts_batch **out);
ts_status ts_batch_destroy(ts_batch *batch);
const char *ts_batch_last_error(const ts_batch *batch);
/* clear every scene's film and restart its passes at first_pass (synchronises) */
ts_status ts_batch_reset(ts_batch *batch, uint32_t first_pass, void *stream);
/* scenes rendered by the next steps: active[num_scenes], nonzero = render (synchronises) */
ts_status ts_batch_set_active(ts_batch *batch, const int32_t *active, void *stream);
/* one step: a block of passes for every active scene, then its block average */
ts_status ts_batch_step(ts_batch *batch, void *stream);
/* error bits raised by the batch's kernels since the last check (synchronises the device) */
ts_status ts_batch_check(ts_batch *batch, uint32_t *bits);

/* ---- device status: error bits raised by kernels since the last call (synchronises) */
ts_status ts_check_device(ts_ctx *ctx, uint32_t *bits);

#ifdef __cplusplus
}
#endif
#endif /* TS_SPECTRAL_H */
