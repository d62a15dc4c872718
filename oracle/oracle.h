/* CPU oracle for the spectral path-tracing hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference renderer's estimator
 * (main.py:682-1629 of Xyzonox/taichi-spectral-render), used by the tests, by
 * the package smoke check and by the CPU-baseline leg of bench.py as the
 * checker.  Nothing in the product links or calls it.
 *
 * Parity status: pinned to the reference's own code.  The reference's
 * estimator is Taichi code and Taichi is not installable here, so its
 * @ti.func functions and its cast_rays kernel were lifted unmodified out of
 * main.py's syntax tree and run in plain Python with float32 arithmetic and
 * given random draws (tests/golden/make_estimator_ref.py); this restatement
 * reproduces their outputs (tests/test_oracle_pinned.py): bit for bit where
 * the arithmetic is +, -, *, /, sqrt (intersect_triangle, intersect_aabb,
 * trace, complex ops, GGX D and G, HG), to the last bits where it calls
 * transcendentals, with identical branch decisions and draw counts, and per
 * film cell to 1e-4 on whole paths of three scenes.  Host preparation (BVH,
 * scene flattening, light CDF, spectral data) is pinned on golden fixtures
 * the reference's host code wrote.  Not reproducible: Taichi's own random
 * stream and its fast-math device intrinsics (last-bit differences).
 *
 * One deliberate departure: a path whose throughput is exactly zero is ended
 * (the reference keeps tracing it; its later deposits are zero, or NaN where
 * a degenerate event computes 0/0 -- e.g. leaving a rough dielectric through
 * an index-matched interface, whose transmission lobe the reference already
 * zeroes on entry because its Smith term clamps the refracted cosine to 0).
 *
 * Everything here follows the reference's data model: triangles and BVH
 * nodes in the reference layout (main.py:255-275), materials as
 * [M][6][B] f32 + [M][2][B] i32 + [M] eem id (main.py:1685-1699), per-band
 * light CDF (main.py:590-627).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t width, height, bands;
  float lambda_min_nm, lambda_step_nm;
  float epsilon, escape;
  int32_t max_path_length, scatter_bounces;
  float aspect_ratio, fov_scale;
  uint32_t seed;
  uint32_t scene_id;  /* mixed into the RNG counter (batched renders) */
} orc_config;

typedef struct {
  /* triangles in BVH (reordered) order, main.py:563-574 */
  int32_t num_tris;
  const float *v0, *v1, *v2, *n0, *n1, *n2, *normal, *area; /* [T][3] / [T] */
  const int32_t *mat_id;
  /* BVH in the reference layout, main.py:576-588 */
  int32_t num_nodes;
  const float *node_min, *node_max; /* [N][3] */
  const int32_t *node_left, *node_right, *node_num_tris, *node_tri_start;
  /* materials, main.py:545-561 */
  int32_t num_materials;
  const float *mat_f32;   /* [M][6][B] */
  const int32_t *mat_i32; /* [M][2][B] */
  const int32_t *mat_eem; /* [M] */
  int32_t num_eems;
  const float *eem; /* [E][B][B], row = excitation band */
  /* lights, main.py:590-627 */
  int32_t max_lights;
  const float *light_cdf;     /* [B][L] */
  const int32_t *light_idx;   /* [B][L] */
  const int32_t *num_lights;  /* [B] */
  const float *light_area;    /* [B] */
  /* camera basis, main.py:633-640 */
  float cam_origin[3], cam_u[3], cam_v[3], cam_w[3];
} orc_scene;

typedef struct {
  int64_t paths, vertices, traces, stack_overflow;
} orc_stats;

/* Philox-4x32-10 block (Salmon et al., SC'11); exposed for the RNG tests. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Single-function known-answer hooks: fresnel_spectral (main.py:925-966),
 * normaldistrobution_ggx (main.py:900-907), evaluate_henyey_greenstein
 * (main.py:758-766), in float32 or float64. */
double orc_fresnel(double cos_i, double ni, double ki, double nt, double kt, int32_t use_double);
double orc_ggx_d(double ndh, double rough, int32_t use_double);
double orc_hg_eval(double cos_t, double g, int32_t use_double);

/* Function-level evaluation (test hook): runs one restated reference function
 * on n rows of inputs, each with its own list of random draws (draw_stride
 * per row; draws may be NULL), FP32.  draws_used[i] = draws row i consumed.
 * Row layouts (in -> out):
 *   TRIANGLE  pos3 dir3 v0_3 v1_3 v2_3            -> t u v   (intersect_triangle, main.py:807-829)
 *   AABB      pos3 inv_dir3 min3 max3              -> hit     (intersect_aabb, main.py:797-805)
 *   TRACE     pos3 dir3  -> t normal3 shading_normal3 mat u v is_hit front tri   (trace, main.py:831-864)
 *   COMPLEX   z.re z.im w.re w.im                  -> sqrt(z) z/w   (main.py:868-896)
 *   FRESNEL   cos_i ni ki nt kt                    -> R       (fresnel_spectral, main.py:925-966)
 *   GGX_D     NdotH roughness                      -> D       (main.py:900-907)
 *   GGX_G     n3 v3 l3 roughness                   -> G       (main.py:909-923)
 *   GGX_SAMPLE xi0 xi1 n3 alpha                    -> h3      (main.py:968-978)
 *   HG        cos g                                -> p       (main.py:758-766)
 *   HG_SAMPLE dir3 g                               -> dir3    (main.py:768-792)
 *   COS_HEMISPHERE n3                              -> dir3    (main.py:689-705)
 *   SPHERE    (none)                               -> dir3    (main.py:682-687)
 *   BSDF      vol surf V3 L3 N3 band               -> bsdf pdf   (evaluate_bsdf, main.py:1360-1444)
 *   SHADOW    origin3 dir3 max_dist light_tri vol band -> T  (shadow_transmittance, main.py:1446-1499)
 *   NEE       pos3 dir3 active transport vol N3 surf -> factor emission weight (main.py:1296-1358)
 *   SURFACE   dir3 active vol hit_mat shading_normal3 -> did_reflect dir3 estimator pdf new_band
 *             (scatter_surface, main.py:1000-1188; ray at the origin)
 *   VOLUME    pos3 dir3 active vol -> action travel estimator normal3 shading_normal3 front hit_mat tri
 *             dir3 new_band penetrated_tri   (scatter_volume, main.py:1190-1292) */
enum {
  ORC_EVAL_TRIANGLE = 0, ORC_EVAL_AABB = 1, ORC_EVAL_TRACE = 2, ORC_EVAL_COMPLEX = 3, ORC_EVAL_FRESNEL = 4,
  ORC_EVAL_GGX_D = 5, ORC_EVAL_GGX_G = 6, ORC_EVAL_GGX_SAMPLE = 7, ORC_EVAL_HG = 8, ORC_EVAL_HG_SAMPLE = 9,
  ORC_EVAL_COS_HEMISPHERE = 10, ORC_EVAL_SPHERE = 11, ORC_EVAL_BSDF = 12, ORC_EVAL_SHADOW = 13, ORC_EVAL_NEE = 14,
  ORC_EVAL_SURFACE = 15, ORC_EVAL_VOLUME = 16
};
void orc_eval(const orc_scene *s, const orc_config *c, int32_t kind, int32_t n, const float *in, int32_t in_stride,
              const float *draws, int32_t draw_stride, float *out, int32_t out_stride, int32_t *draws_used);

/* Closest hit with the reference traversal (main.py:831-864): explicit stack,
 * right child popped first, no distance culling.  rays: [n][6] (pos, dir).
 * Outputs: tri (reordered index, -1 on miss), t (1e9 on miss), u, v. */
void orc_trace(const orc_scene *s, const orc_config *c, const float *rays, int32_t n,
               int32_t *tri, float *t, float *u, float *v, int32_t use_double);

/* Brute-force closest hit over all triangles, ties to the lowest index. */
void orc_trace_brute(const orc_scene *s, const orc_config *c, const float *rays, int32_t n,
                     int32_t *tri, float *t);

/* One sample pass (cast_rays, main.py:1502-1590) for a list of pixels.
 * pixel_ids are j*W+i; deposits are ADDED into out[p*B + band] (double).
 * use_double selects the FP64 estimator.  nthreads<=0: all OpenMP threads. */
void orc_render_pass(const orc_scene *s, const orc_config *c, uint32_t pass_idx, int32_t band,
                     const int32_t *pixel_ids, int32_t npix, double *out, int32_t use_double,
                     int32_t nthreads, orc_stats *stats);

/* Forward-mode adjoint of one pass, in FP64 or FP32 (forward-mode dual numbers
 * through the same estimator, sampled values held fixed and every
 * parameter-dependent sampling decision multiplied by its score factor p/p).
 * param_ids index the material table [M][6][B] followed by the EEM table
 * [E][B][B].  adj: [npix][B] weights of the film deposits.  ADDS
 * sum_p sum_b adj[p][b] * d deposit[p][b] / d param into grad[nparams];
 * out (may be NULL) receives the film of the pass like orc_render_pass. */
void orc_adjoint_pass(const orc_scene *s, const orc_config *c, uint32_t pass_idx, int32_t band,
                      const int32_t *pixel_ids, int32_t npix, const double *adj, int32_t nparams,
                      const int64_t *param_ids, double *grad, double *out, int32_t use_double, int32_t nthreads);

/* The reference SAH builder (build_bvh, main.py:437-507): full sweep over all
 * split positions on 3 axes, leaf at <=10 triangles or when no split beats
 * the leaf cost, flat boxes padded by 1e-6, depth-first node order.  Centroid
 * ties are broken by a stable sort (numpy's argsort order on ties is not
 * specified).  Inputs in original triangle order; outputs the node table and
 * perm[slot] = original index.  Returns the node count or -1 if max_nodes is
 * too small. */
int32_t orc_build_bvh_sweep(int32_t num_tris, const float *v0, const float *v1, const float *v2,
                            int32_t max_nodes, float *node_min, float *node_max, int32_t *left,
                            int32_t *right, int32_t *num_tris_node, int32_t *tri_start,
                            int32_t *perm);

#ifdef __cplusplus
}
#endif
