/* CPU oracle for the spectral path-tracing hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference renderer's estimator
 * (main.py:682-1629 of Xyzonox/taichi-spectral-render), used by the tests, by
 * the package smoke check and by the CPU-baseline leg of bench.py as the
 * checker.  Nothing in the product links or calls it.
 *
 * Parity status: the reference's estimator cannot be executed here (it is
 * Taichi code and Taichi is not installable), so this restatement is pinned
 * only through the reference's own host code (golden BVH / scene / light CDF
 * / spectral data fixtures generated from it) and analytic known answers; the
 * Monte Carlo estimator itself is "parity unpinned" against Taichi's RNG and
 * fast-math codegen.
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
