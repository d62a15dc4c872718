// C ABI of libspectral.so (include/spectral.h): context, scene upload, render
// passes, film operations.  The context owns every device buffer; callers pass
// plain pointers and sizes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bvh.h"
#include "adjoint.cuh"
#include "batch.cuh"
#include "kernels.cuh"
#include "spectral.h"

namespace {

thread_local std::string g_last_error;

constexpr int kMaxBands = 64;
constexpr int kMaxQueueCapacity = 1 << 25;  // wavefront path slots (about 5.5 GB of path state)
constexpr int kDefaultWidth = 2;  // BVH node width when the scene description leaves it at 0

}  // namespace

struct ts_ctx {
  ts_config cfg{};
  ts::DevConfig dc{};
  int num_sms = 0;
  bool has_scene = false;
  ts::DevScene ds{};
  std::vector<void *> scene_allocs;
  std::vector<int32_t> perm;
  ts_scene_info info{};
  float *d_cmf = nullptr;
  double *d_film[3] = {nullptr, nullptr, nullptr};
  int *d_counter = nullptr;
  uint32_t *d_err = nullptr;
  float *d_xyz = nullptr;
  float *d_m9 = nullptr;  // XYZ->RGB matrix for ts_resolve_rgb
  float4 *d_mat = nullptr;  // packed material table (scene allocation), rewritten by ts_update_materials
  float *d_eem = nullptr, *d_qy = nullptr, *d_cdf = nullptr;
  float *d_adj_weight = nullptr;  // adjoint scratch: per-path weighted totals
  size_t adj_weight_cap = 0;      // entries
  ts::WaveBuffers wave{};
  std::vector<void *> wave_allocs;
  ts::WaveLoopGraph *wave_loop = nullptr;  // captured regenerating wavefront loop
  int loop_limit = 0;                      // caller's bound on loop iterations per launch (0 = automatic)
  // path records for the adjoint (ts_record_paths): per path of the armed
  // passes its total deposit, written by megakernel renders of those passes
  float *d_rec = nullptr;
  size_t rec_cap = 0;              // entries allocated
  uint32_t rec_first = 0;          // first pass of the armed range
  int rec_num = 0;                 // passes in the armed range (0 = not armed)
  std::vector<int> rec_band;       // per pass of the range: band it was recorded at (-1 = not recorded)
  size_t film_bytes = 0, scene_bytes = 0, wave_bytes = 0;
  float cam[9] = {0, 0, 3.5f, 0, 0, -1, 0, 1, 0};
  std::string err;
};

namespace {

ts_status fail(ts_ctx *c, ts_status s, const std::string &msg) {
  g_last_error = msg;
  if (c) c->err = msg;
  return s;
}
ts_status cuda_fail(ts_ctx *c, cudaError_t e, const char *what) {
  return fail(c, e == cudaErrorMemoryAllocation ? TS_ERR_OUT_OF_MEMORY : TS_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}
#define TS_CUDA(c, expr, what)                       \
  do {                                               \
    cudaError_t e_ = (expr);                         \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
  } while (0)

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

ts::Film film_of(ts_ctx *c) {
  ts::Film f;
  f.block = c->d_film[TS_FILM_BLOCK];
  f.mean = c->d_film[TS_FILM_MEAN];
  f.m2 = c->d_film[TS_FILM_M2];
  f.W = c->cfg.width;
  f.H = c->cfg.height;
  f.B = c->cfg.bands;
  return f;
}

void free_list(std::vector<void *> &v) {
  for (void *p : v) cudaFree(p);
  v.clear();
}

template <class T>
cudaError_t upload(ts_ctx *c, std::vector<void *> &owner, const T *host, size_t n, T **dev, size_t &bytes) {
  *dev = nullptr;
  const size_t sz = std::max<size_t>(n, 1) * sizeof(T);
  cudaError_t e = cudaMalloc((void **)dev, sz);
  if (e != cudaSuccess) return e;
  owner.push_back(*dev);
  bytes += sz;
  if (n) e = cudaMemcpy(*dev, host, n * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

void camera_basis(const float o[3], const float l[3], const float up[3], float3 &w, float3 &u, float3 &v) {
  // update_camera, main.py:633-640, in float32
  auto norm = [](float3 a) {
    const float n = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return make_float3(a.x / n, a.y / n, a.z / n);
  };
  auto cr = [](float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
  };
  w = norm(make_float3(o[0] - l[0], o[1] - l[1], o[2] - l[2]));
  u = norm(cr(make_float3(up[0], up[1], up[2]), w));
  v = cr(w, u);
}

}  // namespace

extern "C" {

const char *ts_version(void) { return "spectral-b200 0.1 (sm_100a)"; }

const char *ts_last_error(const ts_ctx *ctx) { return ctx ? ctx->err.c_str() : g_last_error.c_str(); }

ts_status ts_create(const ts_config *cfg, ts_ctx **out) {
  if (!cfg || !out) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: null argument");
  *out = nullptr;
  const ts_config &k = *cfg;
  if (k.width <= 0 || k.height <= 0 || (int64_t)k.width * k.height > (1ll << 30))
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: resolution out of range");
  if (k.bands < 1 || k.bands > kMaxBands) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: bands must be 1..64");
  if (k.max_path_length < 0 || k.max_path_length > 1024)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: max_path_length must be 0..1024");
  if (k.scatter_bounces < 1 || k.scatter_bounces > 64)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: scatter_bounces must be 1..64");
  if (k.bands > 1 && !(k.lambda_max_nm > k.lambda_min_nm))
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: lambda_max_nm must exceed lambda_min_nm");
  if (k.kernel != TS_KERNEL_MEGA && k.kernel != TS_KERNEL_WAVEFRONT)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: unknown kernel");
  if (k.traversal != TS_TRAVERSAL_DEFAULT && k.traversal != TS_TRAVERSAL_SPECULATIVE)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: unknown traversal variant");
  if (k.occupancy != 0 && k.occupancy != 5 && k.occupancy != 8)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: occupancy must be 0, 5 or 8");
  if (k.queue_capacity < 0) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: negative queue_capacity");
  if (k.queue_capacity > kMaxQueueCapacity)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: queue_capacity above 2^25 path slots");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(nullptr, TS_ERR_CUDA, "ts_create: no CUDA device");
  if (k.device < 0 || k.device >= ndev) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create: bad device ordinal");
  e = cudaSetDevice(k.device);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
  ts_ctx *c = new ts_ctx();
  c->cfg = k;
  if (c->cfg.block_size <= 0) c->cfg.block_size = 128;
  if (c->cfg.trace_budget <= 0) c->cfg.trace_budget = 32;
  c->cfg.block_size = std::min(ts::kMaxBlock, std::max(32, c->cfg.block_size / 32 * 32));
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, k.device);
  ts::DevConfig &d = c->dc;
  d.W = k.width;
  d.H = k.height;
  d.B = k.bands;
  d.lmin_m = (float)((double)k.lambda_min_nm * 1e-9);
  d.lmin_nm = k.lambda_min_nm;
  d.step_nm = k.bands > 1 ? (float)(((double)k.lambda_max_nm - (double)k.lambda_min_nm) / (k.bands - 1)) : 0.f;
  d.eps = k.epsilon;
  d.escape = k.escape;
  d.max_depth = k.max_path_length;
  d.scatter_bounces = k.scatter_bounces;
  d.aspect = k.aspect_ratio;
  d.fov = k.fov_scale;
  d.seed = k.seed;
  d.scene_id = k.scene_id;
  d.speculative = k.traversal == TS_TRAVERSAL_SPECULATIVE ? 1 : 0;
  const size_t cells = (size_t)k.width * k.height * k.bands;
  for (int i = 0; i < 3; ++i) {
    e = cudaMalloc((void **)&c->d_film[i], cells * sizeof(double));
    if (e != cudaSuccess) {
      ts_destroy(c);
      return cuda_fail(nullptr, e, "ts_create: film allocation");
    }
    cudaMemset(c->d_film[i], 0, cells * sizeof(double));
  }
  c->film_bytes = 3 * cells * sizeof(double);
  e = cudaMalloc((void **)&c->d_counter, 64 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_err, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_xyz, (size_t)k.width * k.height * 3 * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_m9, 9 * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(uint32_t));
  if (e != cudaSuccess) {
    ts_destroy(c);
    return cuda_fail(nullptr, e, "ts_create: allocation");
  }
  *out = c;
  return TS_OK;
}

ts_status ts_set_launch_config(ts_ctx *c, const ts_config *k) {
  if (!c || !k) return fail(c, TS_ERR_INVALID_ARG, "ts_set_launch_config: null argument");
  if (k->kernel != TS_KERNEL_MEGA && k->kernel != TS_KERNEL_WAVEFRONT)
    return fail(c, TS_ERR_INVALID_ARG, "ts_set_launch_config: unknown kernel");
  if (k->traversal != TS_TRAVERSAL_DEFAULT && k->traversal != TS_TRAVERSAL_SPECULATIVE)
    return fail(c, TS_ERR_INVALID_ARG, "ts_set_launch_config: unknown traversal variant");
  if (k->blocks_per_sm < 0 || k->blocks_per_sm > 64 || k->sort_keys < 0 || k->sort_keys > 7 || k->trace_budget < 0)
    return fail(c, TS_ERR_INVALID_ARG, "ts_set_launch_config: launch parameter out of range");
  c->cfg.kernel = k->kernel;
  c->cfg.traversal = k->traversal;
  c->cfg.block_size = std::min(ts::kMaxBlock, std::max(32, (k->block_size > 0 ? k->block_size : 128) / 32 * 32));
  c->cfg.blocks_per_sm = k->blocks_per_sm;
  c->cfg.sort_keys = k->sort_keys;
  if (k->occupancy != 0 && k->occupancy != 5 && k->occupancy != 8)
    return fail(c, TS_ERR_INVALID_ARG, "ts_set_launch_config: occupancy must be 0, 5 or 8");
  c->cfg.trace_budget = k->trace_budget > 0 ? k->trace_budget : 32;
  c->cfg.occupancy = k->occupancy;
  if (k->queue_capacity < 0) return fail(c, TS_ERR_INVALID_ARG, "ts_set_launch_config: negative queue_capacity");
  if (k->queue_capacity > kMaxQueueCapacity)
    return fail(c, TS_ERR_INVALID_ARG, "ts_set_launch_config: queue_capacity above 2^25 path slots");
  c->cfg.queue_capacity = k->queue_capacity;
  c->cfg.loop_host = k->loop_host;
  c->dc.speculative = k->traversal == TS_TRAVERSAL_SPECULATIVE ? 1 : 0;
  return TS_OK;
}

static void rec_invalidate(ts_ctx *c);

ts_status ts_destroy(ts_ctx *c) {
  if (!c) return TS_OK;
  cudaSetDevice(c->cfg.device);
  free_list(c->scene_allocs);
  ts::free_wave_loop(c->wave_loop);
  free_list(c->wave_allocs);
  for (double *p : c->d_film) cudaFree(p);
  cudaFree(c->d_counter);
  cudaFree(c->d_err);
  cudaFree(c->d_xyz);
  cudaFree(c->d_m9);
  cudaFree(c->d_adj_weight);
  cudaFree(c->d_rec);
  delete c;
  return TS_OK;
}

ts_status ts_upload_scene(ts_ctx *c, const ts_scene_desc *sd) {
  if (!c || !sd) return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: null argument");
  rec_invalidate(c);
  cudaSetDevice(c->cfg.device);
  const int T = sd->num_tris, M = sd->num_materials, B = c->cfg.bands, E = sd->num_eems;
  if (T < 0 || (T > 0 && (!sd->v0 || !sd->v1 || !sd->v2 || !sd->n0 || !sd->n1 || !sd->n2 || !sd->normal ||
                          !sd->area || !sd->mat_id)))
    return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: missing triangle arrays");
  if (M <= 0 || !sd->mat_f32 || !sd->mat_i32 || !sd->mat_eem)
    return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: at least one material (air, id 0) is required");
  if (E < 0 || (E > 0 && !sd->eem)) return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: missing EEM table");
  if (!sd->cmf) return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: missing CMF table");
  for (int t = 0; t < T; ++t)
    if (sd->mat_id[t] < 0 || sd->mat_id[t] >= M)
      return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: triangle " + std::to_string(t) + " has material id " +
                                             std::to_string(sd->mat_id[t]) + " outside 0.." +
                                             std::to_string(M - 1));
  for (int m = 0; m < M; ++m)
    if (sd->mat_eem[m] < 0 || (sd->mat_eem[m] > 0 && sd->mat_eem[m] >= E))
      return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: material " + std::to_string(m) + " names EEM " +
                                             std::to_string(sd->mat_eem[m]) + " but only " + std::to_string(E) +
                                             " EEM rows were given");
  for (size_t i = 0; i < (size_t)9 * T; ++i) {
    const float x = (i < (size_t)3 * T ? sd->v0 : (i < (size_t)6 * T ? sd->v1 : sd->v2))[i % (3 * (size_t)T)];
    if (!std::isfinite(x)) return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: non-finite vertex coordinate");
  }

  // ---- BVH
  if (sd->bvh_width != 0 && sd->bvh_width != 2 && sd->bvh_width != 4 && sd->bvh_width != 8)
    return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: bvh_width must be 0, 2, 4 or 8");
  ts::BvhOut bvh;
  std::string err;
  if (sd->bvh_num_nodes > 0) {
    if (!sd->node_min || !sd->node_max || !sd->node_left || !sd->node_right || !sd->node_num_tris ||
        !sd->node_tri_start || !sd->tri_perm)
      return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: incomplete reference BVH");
    if (!ts::bvh_from_reference(T, sd->v0, sd->v1, sd->v2, sd->bvh_num_nodes, sd->node_min, sd->node_max,
                                sd->node_left, sd->node_right, sd->node_num_tris, sd->node_tri_start, sd->tri_perm,
                                bvh, err, sd->bvh_width > 0 ? sd->bvh_width : kDefaultWidth, sd->bvh_quantized != 0))
      return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: " + err);
  } else {
    ts::BvhParams p;
    if (sd->bvh_bins > 0) p.bins = sd->bvh_bins;
    if (sd->bvh_leaf_max > 0) p.leaf_max = std::min(sd->bvh_leaf_max, ts::kLeafMax);
    if (sd->bvh_cost_trav > 0) p.cost_trav = sd->bvh_cost_trav;
    if (sd->bvh_cost_tri > 0) p.cost_tri = sd->bvh_cost_tri;
    p.width = sd->bvh_width > 0 ? sd->bvh_width : kDefaultWidth;
    p.quantize = sd->bvh_quantized != 0;
    if (!ts::build_bvh_binned(T, sd->v0, sd->v1, sd->v2, p, bvh, err))
      return fail(c, TS_ERR_INVALID_ARG, "ts_upload_scene: " + err);
  }

  // ---- triangles in slot order
  std::vector<float4> tri((size_t)3 * T), shade((size_t)3 * T);
  std::vector<int32_t> slot_mat(T);
  for (int s = 0; s < T; ++s) {
    const int o = bvh.perm[s];
    const float *a = sd->v0 + 3 * (size_t)o, *b = sd->v1 + 3 * (size_t)o, *q = sd->v2 + 3 * (size_t)o;
    int32_t oid = o, mid = sd->mat_id[o];
    float fo, fm;
    std::memcpy(&fo, &oid, 4);
    std::memcpy(&fm, &mid, 4);
    tri[3 * s + 0] = make_float4(a[0], a[1], a[2], fo);
    tri[3 * s + 1] = make_float4(b[0] - a[0], b[1] - a[1], b[2] - a[2], fm);
    tri[3 * s + 2] = make_float4(q[0] - a[0], q[1] - a[1], q[2] - a[2], 0.f);
    const float *g = sd->normal + 3 * (size_t)o;
    const float *n0 = sd->n0 + 3 * (size_t)o, *n1 = sd->n1 + 3 * (size_t)o, *n2 = sd->n2 + 3 * (size_t)o;
    shade[3 * s + 0] = make_float4(n0[0], n0[1], n0[2], g[0]);
    shade[3 * s + 1] = make_float4(n1[0], n1[1], n1[2], g[1]);
    shade[3 * s + 2] = make_float4(n2[0], n2[1], n2[2], g[2]);
    slot_mat[s] = mid;
  }
  // ---- materials, main.py:545-561
  std::vector<float4> mat((size_t)M * B * 2);
  for (int m = 0; m < M; ++m)
    for (int b = 0; b < B; ++b) {
      const float *f = sd->mat_f32 + (size_t)m * 6 * B;
      const int32_t *i = sd->mat_i32 + (size_t)m * 2 * B;
      float iv, se;
      std::memcpy(&iv, &i[0 * B + b], 4);
      std::memcpy(&se, &i[1 * B + b], 4);
      mat[((size_t)m * B + b) * 2 + 0] = make_float4(f[0 * B + b], f[1 * B + b], f[2 * B + b], f[3 * B + b]);
      mat[((size_t)m * B + b) * 2 + 1] = make_float4(f[4 * B + b], f[5 * B + b], iv, se);
    }
  // ---- EEM tables: row maximum (quantum yield) and running CDF, float32 in
  // the order the reference's kernels accumulate them (main.py:1247-1272)
  const int Ee = std::max(E, 1);
  std::vector<float> eem((size_t)Ee * B * B, 0.f), qy((size_t)Ee * B, 0.f), cdf((size_t)Ee * B * B, 0.f);
  if (E > 0) std::memcpy(eem.data(), sd->eem, sizeof(float) * (size_t)E * B * B);
  for (int e = 0; e < E; ++e)
    for (int r = 0; r < B; ++r) {
      const float *row = eem.data() + ((size_t)e * B + r) * B;
      float q = 0.f, norm = 0.f;
      for (int j = 0; j < B; ++j) {
        if (row[j] > q) q = row[j];
        norm += row[j];
      }
      qy[(size_t)e * B + r] = q;
      float cum = 0.f;
      for (int j = 0; j < B; ++j) {
        cum += row[j] / norm;
        cdf[((size_t)e * B + r) * B + j] = norm != 0.f ? cum : 0.f;
      }
    }
  // ---- lights per band over slots, main.py:590-627 (float32 sums, CDF left unclamped)
  std::vector<std::vector<int>> lights(B);
  for (int s = 0; s < T; ++s)
    for (int b = 0; b < B; ++b)
      if (sd->mat_i32[(size_t)slot_mat[s] * 2 * B + 1 * B + b]) lights[b].push_back(s);
  int L = 1;
  for (int b = 0; b < B; ++b) L = std::max<int>(L, (int)lights[b].size());
  std::vector<float> lcdf((size_t)B * L, 0.f), larea(B, 0.f);
  std::vector<int32_t> lslot((size_t)B * L, 0), nl(B, 0);
  for (int b = 0; b < B; ++b) {
    nl[b] = (int)lights[b].size();
    if (!nl[b]) continue;
    float tot = 0.f;
    for (int s : lights[b]) tot += sd->area[bvh.perm[s]];
    larea[b] = tot;
    float cum = 0.f;
    for (int i = 0; i < nl[b]; ++i) {
      cum += sd->area[bvh.perm[lights[b][i]]] / tot;
      lcdf[(size_t)b * L + i] = cum;
      lslot[(size_t)b * L + i] = lights[b][i];
    }
  }

  // ---- upload (replace any previous scene)
  free_list(c->scene_allocs);
  c->has_scene = false;
  c->scene_bytes = 0;
  ts::DevScene ds{};
  size_t &by = c->scene_bytes;
  std::vector<void *> &ow = c->scene_allocs;
  float4 *d_node, *d_tri, *d_shade, *d_mat;
  float *d_rmin, *d_rmax, *d_eem, *d_qy, *d_cdf, *d_lcdf, *d_larea, *d_cmf;
  int4 *d_rlink;
  int32_t *d_meem, *d_lslot, *d_nl;
  TS_CUDA(c, upload(c, ow, bvh.node2.data(), bvh.node2.size(), &d_node, by), "upload nodes");
  TS_CUDA(c, upload(c, ow, tri.data(), tri.size(), &d_tri, by), "upload triangles");
  TS_CUDA(c, upload(c, ow, shade.data(), shade.size(), &d_shade, by), "upload normals");
  TS_CUDA(c, upload(c, ow, bvh.ref_min.data(), bvh.ref_min.size(), &d_rmin, by), "upload ref nodes");
  TS_CUDA(c, upload(c, ow, bvh.ref_max.data(), bvh.ref_max.size(), &d_rmax, by), "upload ref nodes");
  TS_CUDA(c, upload(c, ow, bvh.ref_link.data(), bvh.ref_link.size(), &d_rlink, by), "upload ref nodes");
  TS_CUDA(c, upload(c, ow, mat.data(), mat.size(), &d_mat, by), "upload materials");
  TS_CUDA(c, upload(c, ow, sd->mat_eem, (size_t)M, &d_meem, by), "upload materials");
  TS_CUDA(c, upload(c, ow, eem.data(), eem.size(), &d_eem, by), "upload EEM");
  TS_CUDA(c, upload(c, ow, qy.data(), qy.size(), &d_qy, by), "upload EEM");
  TS_CUDA(c, upload(c, ow, cdf.data(), cdf.size(), &d_cdf, by), "upload EEM");
  TS_CUDA(c, upload(c, ow, lcdf.data(), lcdf.size(), &d_lcdf, by), "upload lights");
  TS_CUDA(c, upload(c, ow, lslot.data(), lslot.size(), &d_lslot, by), "upload lights");
  TS_CUDA(c, upload(c, ow, nl.data(), nl.size(), &d_nl, by), "upload lights");
  TS_CUDA(c, upload(c, ow, larea.data(), larea.size(), &d_larea, by), "upload lights");
  TS_CUDA(c, upload(c, ow, sd->cmf, (size_t)3 * B, &d_cmf, by), "upload CMF");
  ds.node = d_node;
  ds.tri = d_tri;
  ds.shade = d_shade;
  ds.node_width = ts::layout_id(bvh.width, bvh.quantized);  // selects the traversal instantiation
  ds.num_nodes = (int)(bvh.node2.size() / ts::node_float4s(bvh.width, bvh.quantized));
  ds.num_tris = T;
  ds.ref_min = d_rmin;
  ds.ref_max = d_rmax;
  ds.ref_link = d_rlink;
  ds.num_ref_nodes = (int)bvh.ref_link.size();
  ds.mat = d_mat;
  c->d_mat = d_mat;
  c->d_eem = d_eem;
  c->d_qy = d_qy;
  c->d_cdf = d_cdf;
  ds.mat_eem = d_meem;
  ds.eem = d_eem;
  ds.eem_qy = d_qy;
  ds.eem_cdf = d_cdf;
  ds.num_materials = M;
  ds.num_eems = E;
  ds.light_cdf = d_lcdf;
  ds.light_slot = d_lslot;
  ds.num_lights = d_nl;
  ds.light_area = d_larea;
  ds.max_lights = L;
  c->ds = ds;
  c->d_cmf = d_cmf;
  c->perm = bvh.perm;
  c->info.num_tris = T;
  c->info.num_nodes = ds.num_nodes;
  c->info.num_ref_nodes = ds.num_ref_nodes;
  c->info.max_depth = bvh.max_depth;
  c->info.leaves = bvh.leaves;
  c->info.sah_cost = bvh.sah_cost;
  c->info.max_lights = L;
  c->info.node_width = bvh.width;
  c->info.node_quantized = bvh.quantized ? 1 : 0;
  c->has_scene = true;
  // keep the current camera basis
  return ts_set_camera(c, c->cam, c->cam + 3, c->cam + 6);
}

ts_status ts_create_view(const ts_ctx *owner, const ts_config *cfg, ts_ctx **out) {
  if (!owner || !cfg || !out) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create_view: null argument");
  *out = nullptr;
  if (!owner->has_scene) return fail(nullptr, TS_ERR_NO_SCENE, "ts_create_view: the owner has no scene uploaded");
  if (cfg->device != owner->cfg.device)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create_view: a view lives on its owner's device");
  if (cfg->bands != owner->cfg.bands || cfg->lambda_min_nm != owner->cfg.lambda_min_nm ||
      cfg->lambda_max_nm != owner->cfg.lambda_max_nm)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_create_view: a view keeps its owner's spectral bands");
  ts_ctx *c = nullptr;
  const ts_status st = ts_create(cfg, &c);
  if (st != TS_OK) return st;
  // the owner's device scene, shared: nothing is uploaded or copied, and the
  // view frees none of it (its scene_allocs stay empty)
  c->ds = owner->ds;
  c->d_mat = owner->d_mat;
  c->d_eem = owner->d_eem;
  c->d_qy = owner->d_qy;
  c->d_cdf = owner->d_cdf;
  c->d_cmf = owner->d_cmf;
  c->perm = owner->perm;
  c->info = owner->info;
  c->has_scene = true;
  const ts_status cs = ts_set_camera(c, owner->cam, owner->cam + 3, owner->cam + 6);
  if (cs != TS_OK) {
    ts_destroy(c);
    return cs;
  }
  *out = c;
  return TS_OK;
}

ts_status ts_scene_info_get(const ts_ctx *c, ts_scene_info *info) {
  if (!c || !info) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_scene_info_get: null argument");
  *info = c->info;
  info->device_bytes = c->scene_bytes + c->film_bytes + c->wave_bytes;
  return TS_OK;
}

ts_status ts_get_tri_perm(const ts_ctx *c, int32_t *perm_out) {
  if (!c || !perm_out) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_get_tri_perm: null argument");
  std::copy(c->perm.begin(), c->perm.end(), perm_out);
  return TS_OK;
}

ts_status ts_build_bvh_host(int32_t T, const float *v0, const float *v1, const float *v2, int32_t bins,
                            int32_t leaf_max, float cost_trav, float cost_tri, int32_t max_nodes, float *nmin,
                            float *nmax, int32_t *left, int32_t *right, int32_t *ntris, int32_t *tstart,
                            int32_t *perm, int32_t *num_nodes_out) {
  if (T < 0 || (T > 0 && (!v0 || !v1 || !v2 || !perm)) || !num_nodes_out)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_build_bvh_host: bad argument");
  ts::BvhParams p;
  if (bins > 0) p.bins = bins;
  if (leaf_max > 0) p.leaf_max = std::min(leaf_max, ts::kLeafMax);
  if (cost_trav > 0) p.cost_trav = cost_trav;
  if (cost_tri > 0) p.cost_tri = cost_tri;
  ts::BvhOut b;
  std::string err;
  if (!ts::build_bvh_binned(T, v0, v1, v2, p, b, err)) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_build_bvh_host: " + err);
  const int N = (int)b.ref_link.size();
  *num_nodes_out = N;
  if (N > max_nodes || (N > 0 && (!nmin || !nmax || !left || !right || !ntris || !tstart)))
    return fail(nullptr, TS_ERR_CAPACITY, "ts_build_bvh_host: output arrays hold " + std::to_string(max_nodes) +
                                              " nodes, " + std::to_string(N) + " needed");
  std::copy(b.ref_min.begin(), b.ref_min.end(), nmin);
  std::copy(b.ref_max.begin(), b.ref_max.end(), nmax);
  for (int i = 0; i < N; ++i) {
    left[i] = b.ref_link[i].x;
    right[i] = b.ref_link[i].y;
    ntris[i] = b.ref_link[i].z;
    tstart[i] = b.ref_link[i].w;
  }
  std::copy(b.perm.begin(), b.perm.end(), perm);
  return TS_OK;
}

ts_status ts_set_camera(ts_ctx *c, const float o[3], const float l[3], const float up[3]) {
  if (!c || !o || !l || !up) return fail(c, TS_ERR_INVALID_ARG, "ts_set_camera: null argument");
  float tmp[9] = {o[0], o[1], o[2], l[0], l[1], l[2], up[0], up[1], up[2]};
  if (std::memcmp(tmp, c->cam, sizeof(tmp)) != 0) rec_invalidate(c);
  std::memcpy(c->cam, tmp, sizeof(tmp));
  float3 w, u, v;
  camera_basis(o, l, up, w, u, v);
  c->ds.cam_o = make_float3(o[0], o[1], o[2]);
  c->ds.cam_u = u;
  c->ds.cam_v = v;
  c->ds.cam_w = w;
  return TS_OK;
}

static ts_status ensure_wave(ts_ctx *c);

// wavefront passes through the regenerating loop: queue_capacity path slots
// (one per pixel when 0)
static ts_status render_wave_loop(ts_ctx *c, uint32_t pass0, int npass, int band0, cudaStream_t st, const char *what) {
  const int64_t npix = (int64_t)c->cfg.width * c->cfg.height;
  const int cap = c->cfg.queue_capacity > 0 ? c->cfg.queue_capacity : (int)npix;
  if (npix * npass + cap > INT32_MAX)
    return fail(c, TS_ERR_CAPACITY, std::string(what) + ": work items plus path slots exceed 2^31");
  const int bs = c->cfg.block_size;
  int per_sm = c->cfg.blocks_per_sm;
  if (per_sm <= 0) per_sm = std::max(1, 2048 / bs);
  TS_CUDA(c, ts::launch_wave_loop(c->ds, c->dc, pass0, band0, npass, film_of(c), c->wave, c->d_err,
                                  c->num_sms * per_sm, bs, st, c->cfg.trace_budget, cap, &c->wave_loop,
                                  c->cfg.loop_host != 0, c->loop_limit),
          what);
  return TS_OK;
}

// ---- path records (ts_record_paths)
// records of passes [p0, p0 + n) when all of them fall inside the armed range
static float *rec_slot(ts_ctx *c, uint32_t p0, int n) {
  if (c->rec_num <= 0) return nullptr;
  const uint32_t off = p0 - c->rec_first;  // unsigned: passes before the range wrap to large offsets
  if (off >= (uint32_t)c->rec_num || (int64_t)off + n > c->rec_num) return nullptr;
  return c->d_rec + (size_t)off * c->cfg.width * c->cfg.height;
}

// every pass of [p0, p0 + n) recorded at the bands an adjoint starting at band0 replays
static bool rec_current(ts_ctx *c, uint32_t p0, int n, int band0) {
  if (!rec_slot(c, p0, n)) return false;
  const uint32_t off = p0 - c->rec_first;
  for (int i = 0; i < n; ++i)
    if (c->rec_band[off + i] != (band0 + i) % c->cfg.bands) return false;
  return true;
}

// anything that changes a pass's paths makes the records stale
static void rec_invalidate(ts_ctx *c) { std::fill(c->rec_band.begin(), c->rec_band.end(), -1); }

// a megakernel launch of npass passes that also writes their path records
static ts_status render_recorded(ts_ctx *c, uint32_t pass0, int npass, int band0, float *rec, cudaStream_t st,
                                 const char *what) {
  const int bs = c->cfg.block_size;
  int per_sm = c->cfg.blocks_per_sm;
  if (per_sm <= 0) per_sm = std::max(1, 2048 / bs);
  ts::Film f = film_of(c);
  f.rec = rec;
  TS_CUDA(c, ts::launch_render_mega(c->ds, c->dc, pass0, band0, f, c->d_counter, c->d_err, c->num_sms * per_sm, bs, st,
                                    nullptr, npass, c->cfg.occupancy),
          what);
  const uint32_t off = pass0 - c->rec_first;
  for (int i = 0; i < npass; ++i) c->rec_band[off + i] = (band0 + i) % c->cfg.bands;
  return TS_OK;
}

ts_status ts_record_paths(ts_ctx *c, uint32_t first_pass, int32_t num_passes) {
  if (!c) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_record_paths: null context");
  if (num_passes < 0) return fail(c, TS_ERR_INVALID_ARG, "ts_record_paths: num_passes must be >= 0");
  c->rec_num = 0;
  c->rec_band.clear();
  if (num_passes == 0) return TS_OK;
  const int64_t need = (int64_t)num_passes * c->cfg.width * c->cfg.height;
  if (need > ((int64_t)1 << 30))
    return fail(c, TS_ERR_CAPACITY, "ts_record_paths: more than 2^30 paths (4 GB of records)");
  cudaSetDevice(c->cfg.device);
  if ((size_t)need > c->rec_cap) {
    cudaFree(c->d_rec);
    c->d_rec = nullptr;
    c->rec_cap = 0;
    TS_CUDA(c, cudaMalloc((void **)&c->d_rec, (size_t)need * sizeof(float)), "ts_record_paths");
    c->rec_cap = (size_t)need;
  }
  c->rec_first = first_pass;
  c->rec_num = num_passes;
  c->rec_band.assign(num_passes, -1);
  return TS_OK;
}

ts_status ts_render_pass(ts_ctx *c, uint32_t pass_idx, int32_t band, void *stream) {
  if (!c) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_render_pass: null context");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_render_pass: no scene uploaded");
  if (band < 0 || band >= c->cfg.bands) return fail(c, TS_ERR_INVALID_ARG, "ts_render_pass: band out of range");
  cudaSetDevice(c->cfg.device);
  const cudaStream_t st = as_stream(stream);
  const int bs = c->cfg.block_size;
  if (float *rec = rec_slot(c, pass_idx, 1)) return render_recorded(c, pass_idx, 1, band, rec, st, "render pass");
  if (c->cfg.kernel == TS_KERNEL_MEGA) {
    int per_sm = c->cfg.blocks_per_sm;
    if (per_sm <= 0) per_sm = std::max(1, 2048 / bs);
    const int grid = c->num_sms * per_sm;
    TS_CUDA(c, ts::launch_render_mega(c->ds, c->dc, pass_idx, band, film_of(c), c->d_counter, c->d_err, grid, bs, st,
                                      nullptr, 1, c->cfg.occupancy),
            "render pass");
  } else {
    ts_status s = ensure_wave(c);
    if (s != TS_OK) return s;
    int per_sm = c->cfg.blocks_per_sm;
    if (per_sm <= 0) per_sm = std::max(1, 2048 / bs);
    const int grid = c->num_sms * per_sm;
    if (c->cfg.queue_capacity > 0 && c->cfg.sort_keys == 0)
      return render_wave_loop(c, pass_idx, 1, band, st, "render pass");
    TS_CUDA(c, ts::launch_wave_pass(c->ds, c->dc, pass_idx, band, film_of(c), c->wave, c->d_err, grid, bs,
                                    c->cfg.sort_keys, st, c->cfg.trace_budget, c->cfg.queue_capacity),
            "render pass");
  }
  return TS_OK;
}

ts_status ts_render_passes(ts_ctx *c, uint32_t first_pass, int32_t num_passes, int32_t first_band, void *stream) {
  if (!c) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_render_passes: null context");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_render_passes: no scene uploaded");
  if (first_band < 0 || first_band >= c->cfg.bands)
    return fail(c, TS_ERR_INVALID_ARG, "ts_render_passes: band out of range");
  if (num_passes < 1 || num_passes > c->cfg.bands)
    return fail(c, TS_ERR_INVALID_ARG, "ts_render_passes: num_passes must be 1..bands (one film plane per pass)");
  if ((int64_t)num_passes * c->cfg.width * c->cfg.height > INT32_MAX)
    return fail(c, TS_ERR_CAPACITY, "ts_render_passes: more than 2^31 paths in one launch");
  if (float *rec = rec_slot(c, first_pass, num_passes)) {
    cudaSetDevice(c->cfg.device);
    return render_recorded(c, first_pass, num_passes, first_band, rec, as_stream(stream), "ts_render_passes");
  }
  if (c->cfg.kernel != TS_KERNEL_MEGA && c->cfg.sort_keys == 0) {
    cudaSetDevice(c->cfg.device);
    const ts_status s = ensure_wave(c);
    if (s != TS_OK) return s;
    return render_wave_loop(c, first_pass, num_passes, first_band, as_stream(stream), "ts_render_passes");
  }
  if (c->cfg.kernel != TS_KERNEL_MEGA) {
    for (int i = 0; i < num_passes; ++i) {
      const ts_status st = ts_render_pass(c, first_pass + (uint32_t)i, (first_band + i) % c->cfg.bands, stream);
      if (st != TS_OK) return st;
    }
    return TS_OK;
  }
  cudaSetDevice(c->cfg.device);
  const int bs = c->cfg.block_size;
  int per_sm = c->cfg.blocks_per_sm;
  if (per_sm <= 0) per_sm = std::max(1, 2048 / bs);
  TS_CUDA(c, ts::launch_render_mega(c->ds, c->dc, first_pass, first_band, film_of(c), c->d_counter, c->d_err,
                                    c->num_sms * per_sm, bs, as_stream(stream), nullptr, num_passes, c->cfg.occupancy),
          "ts_render_passes");
  return TS_OK;
}

ts_status ts_set_loop_iteration_limit(ts_ctx *c, int32_t limit) {
  if (!c) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_set_loop_iteration_limit: null context");
  if (limit < 0) return fail(c, TS_ERR_INVALID_ARG, "ts_set_loop_iteration_limit: limit must be >= 0");
  c->loop_limit = limit;
  return TS_OK;
}

ts_status ts_wave_loop_iterations(ts_ctx *c, void *stream, int32_t *iterations) {
  if (!c || !iterations) return fail(c, TS_ERR_INVALID_ARG, "ts_wave_loop_iterations: null argument");
  *iterations = 0;
  if (!c->wave.loop) return TS_OK;
  cudaSetDevice(c->cfg.device);
  const cudaStream_t st = as_stream(stream);
  TS_CUDA(c, cudaMemcpyAsync(iterations, &c->wave.loop->iter, sizeof(int32_t), cudaMemcpyDeviceToHost, st),
          "ts_wave_loop_iterations");
  TS_CUDA(c, cudaStreamSynchronize(st), "ts_wave_loop_iterations");
  return TS_OK;
}

ts_status ts_render_pass_counted(ts_ctx *c, uint32_t pass_idx, int32_t band, void *stream, uint64_t work[8]) {
  if (!c || !work) return fail(c, TS_ERR_INVALID_ARG, "ts_render_pass_counted: bad argument");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_render_pass_counted: no scene uploaded");
  if (band < 0 || band >= c->cfg.bands) return fail(c, TS_ERR_INVALID_ARG, "ts_render_pass_counted: band out of range");
  cudaSetDevice(c->cfg.device);
  const cudaStream_t st = as_stream(stream);
  const int bs = c->cfg.block_size;
  int per_sm = c->cfg.blocks_per_sm;
  if (per_sm <= 0) per_sm = std::max(1, 2048 / bs);
  unsigned long long *d_work = reinterpret_cast<unsigned long long *>(c->d_counter + 8);
  TS_CUDA(c, cudaMemsetAsync(d_work, 0, 8 * sizeof(unsigned long long), st), "counted pass");
  TS_CUDA(c, ts::launch_render_mega(c->ds, c->dc, pass_idx, band, film_of(c), c->d_counter, c->d_err,
                                    c->num_sms * per_sm, bs, st, d_work),
          "counted pass");
  TS_CUDA(c, cudaMemcpyAsync(work, d_work, 8 * sizeof(uint64_t), cudaMemcpyDeviceToHost, st), "counted pass");
  TS_CUDA(c, cudaStreamSynchronize(st), "counted pass");
  return TS_OK;
}

ts_status ts_render_tile_noalloc(ts_ctx *c, uint32_t pass_idx, int32_t band, int32_t x0, int32_t y0, int32_t tile_w,
                                 int32_t tile_h, double *film_dev, void *stream) {
  if (!c || !film_dev) return fail(c, TS_ERR_INVALID_ARG, "ts_render_tile_noalloc: null argument");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_render_tile_noalloc: no scene uploaded");
  if (band < 0 || band >= c->cfg.bands) return fail(c, TS_ERR_INVALID_ARG, "ts_render_tile_noalloc: band out of range");
  if (tile_w <= 0 || tile_h <= 0 || x0 < 0 || y0 < 0 || x0 > c->cfg.width - tile_w || y0 > c->cfg.height - tile_h)
    return fail(c, TS_ERR_INVALID_ARG, "ts_render_tile_noalloc: tile outside the frame");
  const int64_t n = (int64_t)tile_w * tile_h;
  if (n > ts::noalloc_max_paths())
    return fail(c, TS_ERR_CAPACITY, "ts_render_tile_noalloc: a tile of " + std::to_string(n) +
                                        " pixels exceeds the allocation-free limit of " +
                                        std::to_string(ts::noalloc_max_paths()) + " pixels per call");
  TS_CUDA(c, cudaSetDevice(c->cfg.device), "ts_render_tile_noalloc");
  void *scratch = nullptr;
  TS_CUDA(c, ts::noalloc_setup(c->cfg.device, &scratch), "ts_render_tile_noalloc: scratch address lookup");
  ts::Film f;
  f.block = film_dev;
  f.mean = nullptr;
  f.m2 = nullptr;
  f.W = c->cfg.width;
  f.H = c->cfg.height;
  f.B = c->cfg.bands;
  const int bs = c->cfg.block_size;
  int per_sm = c->cfg.blocks_per_sm;
  if (per_sm <= 0) per_sm = std::max(1, 2048 / bs);
  TS_CUDA(c, ts::launch_wave_tile_noalloc(c->ds, c->dc, pass_idx, band, f, scratch, x0, y0, tile_w, tile_h, c->d_err,
                                          c->num_sms * per_sm, bs, as_stream(stream), c->cfg.trace_budget),
          "ts_render_tile_noalloc");
  return TS_OK;
}

ts_status ts_accumulate_block(ts_ctx *c, int32_t n, void *stream) {
  if (!c) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_accumulate_block: null context");
  if (n < 1) return fail(c, TS_ERR_INVALID_ARG, "ts_accumulate_block: num_blocks_completed must be >= 1");
  cudaSetDevice(c->cfg.device);
  TS_CUDA(c, ts::launch_accumulate_block(film_of(c), n, as_stream(stream)), "accumulate");
  return TS_OK;
}

ts_status ts_reset(ts_ctx *c, void *stream) {
  if (!c) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_reset: null context");
  cudaSetDevice(c->cfg.device);
  TS_CUDA(c, ts::launch_clear_film(film_of(c), as_stream(stream)), "reset");
  return TS_OK;
}

ts_status ts_film_buffer(ts_ctx *c, int32_t which, double **dev_ptr, size_t *count) {
  if (!c || !dev_ptr || !count || which < 0 || which > 2)
    return fail(c, TS_ERR_INVALID_ARG, "ts_film_buffer: bad argument");
  *dev_ptr = c->d_film[which];
  *count = (size_t)c->cfg.width * c->cfg.height * c->cfg.bands;
  return TS_OK;
}

ts_status ts_film_download(ts_ctx *c, int32_t which, double *host, void *stream) {
  if (!c || !host || which < 0 || which > 2) return fail(c, TS_ERR_INVALID_ARG, "ts_film_download: bad argument");
  cudaSetDevice(c->cfg.device);
  const size_t n = (size_t)c->cfg.width * c->cfg.height * c->cfg.bands;
  TS_CUDA(c, cudaMemcpyAsync(host, c->d_film[which], n * sizeof(double), cudaMemcpyDeviceToHost, as_stream(stream)),
          "film download");
  TS_CUDA(c, cudaStreamSynchronize(as_stream(stream)), "film download");
  return TS_OK;
}

ts_status ts_resolve_xyz(ts_ctx *c, double scale, float *xyz_dev, void *stream) {
  if (!c || !xyz_dev) return fail(c, TS_ERR_INVALID_ARG, "ts_resolve_xyz: bad argument");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_resolve_xyz: no scene (CMF) uploaded");
  cudaSetDevice(c->cfg.device);
  TS_CUDA(c, ts::launch_resolve_xyz(film_of(c), c->d_cmf, scale, xyz_dev, as_stream(stream)), "resolve xyz");
  return TS_OK;
}

ts_status ts_resolve_xyz_host(ts_ctx *c, double scale, float *xyz_host, void *stream) {
  if (!c || !xyz_host) return fail(c, TS_ERR_INVALID_ARG, "ts_resolve_xyz_host: bad argument");
  ts_status s = ts_resolve_xyz(c, scale, c->d_xyz, stream);
  if (s != TS_OK) return s;
  const size_t n = (size_t)c->cfg.width * c->cfg.height * 3;
  TS_CUDA(c, cudaMemcpyAsync(xyz_host, c->d_xyz, n * sizeof(float), cudaMemcpyDeviceToHost, as_stream(stream)),
          "resolve xyz copy");
  TS_CUDA(c, cudaStreamSynchronize(as_stream(stream)), "resolve xyz sync");
  return TS_OK;
}

ts_status ts_resolve_rgb(ts_ctx *c, double scale, const float M[9], float exposure, float gamma, int32_t iw,
                         int32_t ih, float *rgb_dev, void *stream) {
  if (!c || !M || !rgb_dev || iw <= 0 || ih <= 0) return fail(c, TS_ERR_INVALID_ARG, "ts_resolve_rgb: bad argument");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_resolve_rgb: no scene (CMF) uploaded");
  cudaSetDevice(c->cfg.device);
  TS_CUDA(c, cudaMemcpyAsync(c->d_m9, M, 9 * sizeof(float), cudaMemcpyHostToDevice, as_stream(stream)),
          "resolve rgb matrix");
  TS_CUDA(c, ts::launch_resolve_rgb(film_of(c), c->d_cmf, scale, c->d_m9, exposure, gamma, iw, ih, rgb_dev,
                                    as_stream(stream)),
          "resolve rgb");
  return TS_OK;
}

ts_status ts_trace_batch(ts_ctx *c, const float *rays, int32_t n, int32_t mode, int32_t *tri, float *t, float *u,
                         float *v, void *stream) {
  if (!c || n < 0 || (n > 0 && (!rays || !tri || !t))) return fail(c, TS_ERR_INVALID_ARG, "ts_trace_batch: bad argument");
  if (mode != TS_TRACE_FAST && mode != TS_TRACE_REFERENCE_ORDER)
    return fail(c, TS_ERR_INVALID_ARG, "ts_trace_batch: unknown mode");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_trace_batch: no scene uploaded");
  cudaSetDevice(c->cfg.device);
  TS_CUDA(c, ts::launch_trace_batch(c->ds, c->dc.eps, rays, n, mode, tri, t, u, v, c->d_err, as_stream(stream)),
          "trace batch");
  return TS_OK;
}

ts_status ts_render_normals(ts_ctx *c, float *out, void *stream) {
  if (!c || !out) return fail(c, TS_ERR_INVALID_ARG, "ts_render_normals: bad argument");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_render_normals: no scene uploaded");
  cudaSetDevice(c->cfg.device);
  TS_CUDA(c, ts::launch_render_normals(c->ds, c->dc, out, c->d_err, as_stream(stream)), "render normals");
  return TS_OK;
}

ts_status ts_param_count(const ts_ctx *c, int64_t *num_material_params, int64_t *num_eem_params) {
  if (!c || !num_material_params || !num_eem_params)
    return fail(nullptr, TS_ERR_INVALID_ARG, "ts_param_count: null argument");
  if (!c->has_scene) return fail(const_cast<ts_ctx *>(c), TS_ERR_NO_SCENE, "ts_param_count: no scene uploaded");
  const int64_t B = c->cfg.bands;
  *num_material_params = (int64_t)c->ds.num_materials * 6 * B;
  *num_eem_params = (int64_t)c->ds.num_eems * B * B;
  return TS_OK;
}

ts_status ts_update_materials(ts_ctx *c, const float *mat_f32_dev, const float *eem_dev, void *stream) {
  if (!c) return fail(nullptr, TS_ERR_INVALID_ARG, "ts_update_materials: null context");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_update_materials: no scene uploaded");
  if (eem_dev && c->ds.num_eems <= 0)
    return fail(c, TS_ERR_INVALID_ARG, "ts_update_materials: the scene has no EEM table");
  cudaSetDevice(c->cfg.device);
  rec_invalidate(c);
  TS_CUDA(c, ts::launch_update_materials(c->d_mat, mat_f32_dev, c->ds.num_materials, c->cfg.bands, c->d_eem, c->d_qy,
                                         c->d_cdf, eem_dev, c->ds.num_eems, as_stream(stream)),
          "ts_update_materials");
  return TS_OK;
}

ts_status ts_adjoint_pass(ts_ctx *c, uint32_t pass_idx, int32_t band, const double *adj_dev, double *grad_dev,
                          void *stream) {
  return ts_adjoint_passes(c, pass_idx, 1, band, adj_dev, grad_dev, stream);
}

ts_status ts_adjoint_passes(ts_ctx *c, uint32_t first_pass, int32_t num_passes, int32_t band, const double *adj_dev,
                            double *grad_dev, void *stream) {
  if (!c || !adj_dev || !grad_dev) return fail(c, TS_ERR_INVALID_ARG, "ts_adjoint_pass: null argument");
  if (!c->has_scene) return fail(c, TS_ERR_NO_SCENE, "ts_adjoint_pass: no scene uploaded");
  if (band < 0 || band >= c->cfg.bands) return fail(c, TS_ERR_INVALID_ARG, "ts_adjoint_pass: band out of range");
  if (num_passes < 1) return fail(c, TS_ERR_INVALID_ARG, "ts_adjoint_passes: num_passes must be positive");
  if ((int64_t)num_passes * c->cfg.width * c->cfg.height > INT32_MAX)
    return fail(c, TS_ERR_CAPACITY, "ts_adjoint_passes: more than 2^31 paths in one launch");
  if (c->cfg.scatter_bounces > ts::kAdjMaxSeg)
    return fail(c, TS_ERR_INVALID_ARG, "ts_adjoint_pass: scatter_bounces above " + std::to_string(ts::kAdjMaxSeg) +
                                           " is not supported by the adjoint");
  cudaSetDevice(c->cfg.device);
  const int grid = c->num_sms * 4;
  // the two replays pass each path's weighted total through device scratch;
  // launches are chunked so that it stays <= 64 MB
  const int64_t npix = (int64_t)c->cfg.width * c->cfg.height;
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(num_passes, ts::kAdjMaxPathsPerLaunch / npix));
  const size_t need = (size_t)(chunk * npix);
  if (need > c->adj_weight_cap) {
    cudaFree(c->d_adj_weight);
    c->d_adj_weight = nullptr;
    c->adj_weight_cap = 0;
    TS_CUDA(c, cudaMalloc((void **)&c->d_adj_weight, need * sizeof(float)), "ts_adjoint_pass: scratch");
    c->adj_weight_cap = need;
  }
  for (int64_t p0 = 0; p0 < num_passes; p0 += chunk) {
    const int n = (int)std::min<int64_t>(chunk, num_passes - p0);
    const uint32_t cp = first_pass + (uint32_t)p0;
    const int cb = (int)((band + p0) % c->cfg.bands);
    // paths the forward pass recorded skip the weight replay
    const float *rec = rec_current(c, cp, n, cb) ? rec_slot(c, cp, n) : nullptr;
    TS_CUDA(c, ts::launch_adjoint(c->ds, c->dc, cp, cb, adj_dev, grad_dev, c->d_adj_weight, c->d_counter, c->d_err,
                                  grid, as_stream(stream), n, rec),
            "ts_adjoint_pass");
  }
  return TS_OK;
}

ts_status ts_check_device(ts_ctx *c, uint32_t *bits) {
  if (!c || !bits) return fail(c, TS_ERR_INVALID_ARG, "ts_check_device: bad argument");
  cudaSetDevice(c->cfg.device);
  TS_CUDA(c, cudaDeviceSynchronize(), "device synchronise");
  TS_CUDA(c, cudaMemcpy(bits, c->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost), "read device status");
  TS_CUDA(c, cudaMemset(c->d_err, 0, sizeof(uint32_t)), "clear device status");
  if (*bits) {
    std::string m = "device reported:";
    if (*bits & ts::kErrStackOverflow) m += " traversal stack overflow;";
    if (*bits & ts::kErrQueueOverflow) m += " queue overflow;";
    if (*bits & ts::kErrIterationCap) m += " iteration cap reached;";
    return fail(c, TS_ERR_DEVICE_FAULT, m);
  }
  return TS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- batches
static cudaError_t alloc_wave_buffers(ts::WaveBuffers &w, std::vector<void *> &allocs, size_t &bytes, int n,
                                      bool views);

struct ts_batch {
  int device = 0, n = 0, width = 2;
  ts_batch_config cfg{};
  int num_sms = 0;
  std::vector<ts_ctx *> ctxs;
  std::vector<ts::BatchSlot> host;
  std::vector<int32_t> active;  // per slot
  std::vector<int> order;       // slot k renders the caller's scene order[k]
  ts::BatchSlot *d_slots = nullptr;
  ts::BatchHeader *d_hdr = nullptr;
  int *d_active = nullptr;
  uint32_t *d_err = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // batch loop (cfg.kernel == TS_KERNEL_WAVEFRONT): path state over queue_capacity slots
  ts::WaveBuffers wave{};
  std::vector<void *> wave_allocs;
  size_t wave_bytes = 0;
  ts::BatchLoopGraph *loop = nullptr;
  int loop_cap = 0, loop_limit = 0;
  std::string err;
};

namespace {
ts_status bfail(ts_batch *b, ts_status s, const std::string &msg) {
  g_last_error = msg;
  if (b) b->err = msg;
  return s;
}
#define TS_BCUDA(b, expr, what)                                                             \
  do {                                                                                      \
    cudaError_t e_ = (expr);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return bfail(b, e_ == cudaErrorMemoryAllocation ? TS_ERR_OUT_OF_MEMORY : TS_ERR_CUDA, \
                   std::string(what) + ": " + cudaGetErrorString(e_));                      \
  } while (0)

void batch_free(ts_batch *b) {
  ts::free_batch_loop(b->loop);
  b->loop = nullptr;
  for (void *p : b->wave_allocs) cudaFree(p);
  b->wave_allocs.clear();
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap) cudaStreamDestroy(b->cap);
  cudaFree(b->d_slots);
  cudaFree(b->d_hdr);
  cudaFree(b->d_active);
  cudaFree(b->d_err);
}

int batch_width(const ts_ctx *c) { return c->ds.node_width == 2 && c->dc.speculative ? 3 : c->ds.node_width; }
}  // namespace

extern "C" {

ts_status ts_batch_create(const ts_batch_config *cfg, ts_ctx *const *ctxs, int32_t n, ts_batch **out) {
  if (!ctxs || !out) return bfail(nullptr, TS_ERR_INVALID_ARG, "ts_batch_create: null argument");
  *out = nullptr;
  if (n < 1 || n > ts::kBatchMaxScenes)
    return bfail(nullptr, TS_ERR_INVALID_ARG,
                 "ts_batch_create: 1.." + std::to_string(ts::kBatchMaxScenes) + " scenes per batch");
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i] || !ctxs[i]->has_scene)
      return bfail(nullptr, TS_ERR_NO_SCENE, "ts_batch_create: scene " + std::to_string(i) + " has no scene uploaded");
    if (ctxs[i]->cfg.device != ctxs[0]->cfg.device)
      return bfail(nullptr, TS_ERR_INVALID_ARG, "ts_batch_create: all scenes must live on one device");
    if (batch_width(ctxs[i]) != batch_width(ctxs[0]))
      return bfail(nullptr, TS_ERR_INVALID_ARG,
                   "ts_batch_create: all scenes of a batch need the same BVH width and traversal variant");
  }
  if (cfg && cfg->kernel != TS_KERNEL_MEGA && cfg->kernel != TS_KERNEL_WAVEFRONT)
    return bfail(nullptr, TS_ERR_INVALID_ARG, "ts_batch_create: kernel must be TS_KERNEL_MEGA or TS_KERNEL_WAVEFRONT");
  if (cfg && (cfg->queue_capacity < 0 || cfg->queue_capacity > (1 << 25)))
    return bfail(nullptr, TS_ERR_INVALID_ARG, "ts_batch_create: queue_capacity must be 0..2^25");
  {
    int64_t total = 0;
    for (int i = 0; i < n; ++i) total += (int64_t)ctxs[i]->cfg.bands * ctxs[i]->cfg.width * ctxs[i]->cfg.height;
    if (total + (1 << 25) > INT32_MAX)
      return bfail(nullptr, TS_ERR_CAPACITY, "ts_batch_create: more than 2^31 paths per step");
  }
  ts_batch *b = new ts_batch();
  b->device = ctxs[0]->cfg.device;
  b->n = n;
  b->width = batch_width(ctxs[0]);
  if (cfg) b->cfg = *cfg;
  if (b->cfg.block_size <= 0) b->cfg.block_size = 128;
  b->cfg.block_size = std::min(128, std::max(32, b->cfg.block_size / 32 * 32));
  if (b->cfg.blocks_per_sm <= 0) b->cfg.blocks_per_sm = 5;  // the render kernel's resident blocks per SM
  if (b->cfg.kernel == TS_KERNEL_WAVEFRONT && b->cfg.queue_capacity <= 0) b->cfg.queue_capacity = 1 << 24;
  if (b->cfg.trace_budget <= 0) b->cfg.trace_budget = 16;
  cudaSetDevice(b->device);
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
  // Work-pool order: deepest scenes first (then larger frames), so that a
  // step drains on the shortest paths instead of idling behind the longest.
  b->order.resize(n);
  for (int i = 0; i < n; ++i) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
    const ts::DevConfig &a = ctxs[x]->dc, &c = ctxs[y]->dc;
    if (a.max_depth != c.max_depth) return a.max_depth > c.max_depth;
    return (int64_t)a.W * a.H > (int64_t)c.W * c.H;
  });
  b->ctxs.resize(n);
  for (int k = 0; k < n; ++k) b->ctxs[k] = ctxs[b->order[k]];
  b->host.resize(n);
  b->active.assign(n, 1);
  for (int k = 0; k < n; ++k) {
    ts::BatchSlot &sl = b->host[k];
    std::memset(&sl, 0, sizeof(sl));
    sl.s = b->ctxs[k]->ds;
    sl.c = b->ctxs[k]->dc;
    sl.f = film_of(b->ctxs[k]);
    sl.active = 1;
  }
  cudaError_t e = cudaMalloc((void **)&b->d_slots, sizeof(ts::BatchSlot) * n);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_hdr, sizeof(ts::BatchHeader));
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_active, sizeof(int) * n);
  if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_err, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_slots, b->host.data(), sizeof(ts::BatchSlot) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_active, b->active.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = ts::batch_set_smem_limit(n);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
  if (e == cudaSuccess && b->cfg.kernel == TS_KERNEL_WAVEFRONT) {
    // path slots of the loop: the step's work items (all scenes active), at most queue_capacity
    int64_t total = 0;
    int depth = 0;
    for (int k = 0; k < n; ++k) {
      const ts::DevConfig &c = b->host[k].c;
      total += (int64_t)c.B * c.W * c.H;
      depth = std::max(depth, c.max_depth);
    }
    const int64_t cap = std::max<int64_t>(1, std::min<int64_t>(total, b->cfg.queue_capacity));
    // every slot starts a new item at least once per max_depth iterations while items are left
    const int64_t bound = ((total + cap - 1) / cap + 2) * (int64_t)(depth + 1) + 4;
    b->loop_cap = (int)cap;
    b->loop_limit = (int)std::min<int64_t>(bound, INT32_MAX);
    e = alloc_wave_buffers(b->wave, b->wave_allocs, b->wave_bytes, b->loop_cap, true);
  }
  if (e != cudaSuccess) {
    const std::string msg = std::string("ts_batch_create: ") + cudaGetErrorString(e);
    batch_free(b);
    delete b;
    return bfail(nullptr, e == cudaErrorMemoryAllocation ? TS_ERR_OUT_OF_MEMORY : TS_ERR_CUDA, msg);
  }
  *out = b;
  return TS_OK;
}

ts_status ts_batch_destroy(ts_batch *b) {
  if (!b) return TS_OK;
  cudaSetDevice(b->device);
  batch_free(b);
  delete b;
  return TS_OK;
}

const char *ts_batch_last_error(const ts_batch *b) { return b ? b->err.c_str() : g_last_error.c_str(); }

ts_status ts_batch_reset(ts_batch *b, uint32_t first_pass, void *stream) {
  if (!b) return bfail(nullptr, TS_ERR_INVALID_ARG, "ts_batch_reset: null batch");
  cudaSetDevice(b->device);
  const cudaStream_t st = as_stream(stream);
  for (int i = 0; i < b->n; ++i) {
    TS_BCUDA(b, ts::launch_clear_film(film_of(b->ctxs[i]), st), "ts_batch_reset");
    b->host[i].pass0 = first_pass;
    b->host[i].nblocks = 0;
    b->host[i].active = b->active[i];
  }
  TS_BCUDA(b, cudaMemcpyAsync(b->d_slots, b->host.data(), sizeof(ts::BatchSlot) * b->n, cudaMemcpyHostToDevice, st),
           "ts_batch_reset");
  TS_BCUDA(b, cudaStreamSynchronize(st), "ts_batch_reset");
  return TS_OK;
}

ts_status ts_batch_set_active(ts_batch *b, const int32_t *active, void *stream) {
  if (!b || !active) return bfail(b, TS_ERR_INVALID_ARG, "ts_batch_set_active: null argument");
  cudaSetDevice(b->device);
  for (int k = 0; k < b->n; ++k) b->active[k] = active[b->order[k]] ? 1 : 0;
  TS_BCUDA(b, cudaMemcpyAsync(b->d_active, b->active.data(), sizeof(int) * b->n, cudaMemcpyHostToDevice,
                              as_stream(stream)),
           "ts_batch_set_active");
  TS_BCUDA(b, cudaStreamSynchronize(as_stream(stream)), "ts_batch_set_active");
  return TS_OK;
}

ts_status ts_batch_step(ts_batch *b, void *stream) {
  if (!b) return bfail(nullptr, TS_ERR_INVALID_ARG, "ts_batch_step: null batch");
  cudaSetDevice(b->device);
  const int grid = b->num_sms * b->cfg.blocks_per_sm;
  const int acc_blocks = b->num_sms * 2;
  if (b->cfg.kernel == TS_KERNEL_WAVEFRONT) {
    // one regenerating wavefront loop over every active scene's block; with
    // use_graph the whole step (prepare, init, while-loop, averages) is one graph
    TS_BCUDA(b, ts::launch_batch_loop_step(b->d_slots, b->n, b->d_hdr, b->d_active, b->d_err, b->wave, b->width,
                                           b->num_sms * 8, ts::kMaxBlock, b->cfg.trace_budget, b->loop_cap,
                                           b->loop_limit, acc_blocks, as_stream(stream), &b->loop,
                                           b->cfg.use_graph != 0),
             "ts_batch_step");
    return TS_OK;
  }
  if (!b->cfg.use_graph) {
    TS_BCUDA(b, ts::launch_batch_step(b->d_slots, b->n, b->d_hdr, b->d_active, b->d_err, b->width, grid,
                                      b->cfg.block_size, acc_blocks, as_stream(stream), b->cfg.occupancy),
             "ts_batch_step");
    return TS_OK;
  }
  if (!b->exec) {
    TS_BCUDA(b, cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "ts_batch_step: capture");
    const cudaError_t le = ts::launch_batch_step(b->d_slots, b->n, b->d_hdr, b->d_active, b->d_err, b->width, grid,
                                                 b->cfg.block_size, acc_blocks, b->cap, b->cfg.occupancy);
    const cudaError_t ce = cudaStreamEndCapture(b->cap, &b->graph);
    TS_BCUDA(b, le, "ts_batch_step: capture");
    TS_BCUDA(b, ce, "ts_batch_step: capture");
    TS_BCUDA(b, cudaGraphInstantiate(&b->exec, b->graph, 0), "ts_batch_step: graph instantiation");
  }
  TS_BCUDA(b, cudaGraphLaunch(b->exec, as_stream(stream)), "ts_batch_step: graph launch");
  return TS_OK;
}

ts_status ts_batch_check(ts_batch *b, uint32_t *bits) {
  if (!b || !bits) return bfail(b, TS_ERR_INVALID_ARG, "ts_batch_check: null argument");
  cudaSetDevice(b->device);
  TS_BCUDA(b, cudaDeviceSynchronize(), "ts_batch_check");
  TS_BCUDA(b, cudaMemcpy(bits, b->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost), "ts_batch_check");
  TS_BCUDA(b, cudaMemset(b->d_err, 0, sizeof(uint32_t)), "ts_batch_check");
  if (*bits)
    return bfail(b, TS_ERR_DEVICE_FAULT, "ts_batch_check: a kernel reported error bits " + std::to_string(*bits));
  return TS_OK;
}

}  // extern "C"

// path-state buffers of the wavefront renderers: n slots (views: also the
// per-slot and per-query batch view arrays of the batch loop)
static cudaError_t alloc_wave_buffers(ts::WaveBuffers &w, std::vector<void *> &allocs, size_t &bytes, int n,
                                      bool views) {
  auto grab = [&](void **p, size_t b) -> cudaError_t {
    cudaError_t e = cudaMalloc(p, b);
    if (e == cudaSuccess) {
      allocs.push_back(*p);
      bytes += b;
    }
    return e;
  };
  const size_t N = (size_t)n;
  cudaError_t e = cudaSuccess;
  for (auto *p : {(void **)&w.pos_thr, (void **)&w.dir_spdf, (void **)&w.hit, (void **)&w.sq_origin,
                  (void **)&w.sq_dir})
    if (e == cudaSuccess) e = grab(p, N * sizeof(float4));
  for (auto *p : {(void **)&w.meta, (void **)&w.sq_meta})
    if (e == cudaSuccess) e = grab(p, N * sizeof(int4));
  for (auto *p : {(void **)&w.queue[0], (void **)&w.queue[1], (void **)&w.shadow_queue, (void **)&w.sorted,
                  (void **)&w.trace_order, (void **)&w.shadow_order, (void **)&w.tag})
    if (e == cudaSuccess) e = grab(p, N * sizeof(int));
  if (views) {
    for (auto *p : {(void **)&w.view, (void **)&w.sq_view})
      if (e == cudaSuccess) e = grab(p, N * sizeof(int));
  }
  if (e == cudaSuccess) e = grab((void **)&w.counts, 8192 * sizeof(int));
  if (e == cudaSuccess) e = grab((void **)&w.key_hist, 2 * ts::kMaxKeys * sizeof(int));
  if (e == cudaSuccess) e = grab((void **)&w.loop, sizeof(ts::WaveLoop));
  if (e == cudaSuccess) e = cudaMemset(w.loop, 0, sizeof(ts::WaveLoop));
  if (e == cudaSuccess) w.capacity = n;
  return e;
}

// wavefront buffers are created on first use (one slot per pixel)
static ts_status ensure_wave(ts_ctx *c) {
  const int npix = c->cfg.width * c->cfg.height;
  const int n = c->cfg.queue_capacity > 0 ? c->cfg.queue_capacity : npix;
  if (c->wave.capacity >= n) return TS_OK;
  free_list(c->wave_allocs);
  c->wave = ts::WaveBuffers{};
  c->wave_bytes = 0;
  TS_CUDA(c, alloc_wave_buffers(c->wave, c->wave_allocs, c->wave_bytes, n, false), "wavefront buffers");
  return TS_OK;
}
