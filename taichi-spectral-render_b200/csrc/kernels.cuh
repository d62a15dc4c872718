// Host-side launchers of the device kernels (implemented in *.cu files).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace ts {

// Film layout: [band][row j][column i] FP64, band-major so that one warp of
// neighbouring pixels depositing into the same band writes 256 contiguous bytes.
struct Film {
  double *block;  // current block's per-band sums (block_accumulator)
  double *mean;   // running mean over completed blocks (spectral_accumulator)
  double *m2;     // sum over blocks of block^2 (for the per-pixel standard error)
  int W, H, B;
  // path records for the adjoint (megakernel only; nullptr = none): per work
  // item of the launch the path's total deposit, or -1 where volume
  // fluorescence moved the path to another band
  float *rec = nullptr;
};

// npass consecutive sample passes (cast_rays) from pass / band, band wrapping
// mod B (npass <= B): persistent megakernel with per-lane path regeneration.
// work != nullptr selects the counting variant (work[8], accumulated)
cudaError_t launch_render_mega(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                               int *counter, uint32_t *err, int grid, int block, cudaStream_t st,
                               unsigned long long *work = nullptr, int npass = 1, int occupancy = 0);

// closest hit for a ray batch; mode 0 = fast traversal, 1 = reference order
cudaError_t launch_trace_batch(const DevScene &s, float eps, const float *rays, int n, int mode, int32_t *tri_orig,
                               float *t, float *u, float *v, uint32_t *err, cudaStream_t st);

cudaError_t launch_accumulate_block(Film f, int num_blocks_completed, cudaStream_t st);
cudaError_t launch_clear_film(Film f, cudaStream_t st);
cudaError_t launch_resolve_xyz(Film f, const float *cmf, double scale, float *xyz, cudaStream_t st);
cudaError_t launch_resolve_rgb(Film f, const float *cmf, double scale, const float *xyz_to_rgb, float exposure,
                               float gamma, int img_w, int img_h, float *rgb, cudaStream_t st);
cudaError_t launch_render_normals(const DevScene &s, const DevConfig &c, float *out, uint32_t *err,
                                  cudaStream_t st);

// ---- wavefront renderer -------------------------------------------------------
// state of the regenerating wavefront loop (render_wave.cu), device memory
struct WaveLoop {
  int ext[2];     // extension queue lengths: queue[a] is traced at the iterations of parity a
  int sh[2];      // shadow queries appended by the shade of parity a
  int fetch[2];   // trace / shade work counters of the current iteration
  int next_item;  // next work item (pass offset * npix + pixel) to start
  int total;      // work items of the launch
  int iter, limit;
  uint32_t pass0;
  int band0, shared, pad_;
  float3 cam_o, cam_u, cam_v, cam_w;  // the camera of the launch (not captured in the loop graph)
  int go;                             // continue flag of the last iteration
};

struct WaveBuffers {
  // path state, one slot per pixel
  float4 *pos_thr;    // pos.xyz, throughput
  float4 *dir_spdf;   // dir.xyz, surface pdf
  int4 *meta;         // (pixel, active | active_px << 8 | plen << 16, vol, rng draw index)
  float4 *hit;        // (t, u, v, slot bits) of the last extension trace
  // shadow queries, one slot per queued path
  float4 *sq_origin;  // origin.xyz, max_dist
  float4 *sq_dir;     // dir.xyz, contrib
  int4 *sq_meta;      // (pixel, light_slot, vol, band)
  int *queue[2];      // extension queues (ping-pong), path ids
  int *shadow_queue;  // shadow queue, query ids == path ids
  int *sorted;        // extension queue ordered by material key (shading)
  int *trace_order;   // extension queue ordered by direction octant (tracing)
  int *shadow_order;  // shadow query indices ordered by light triangle
  int *counts;        // [2*max_depth + 8]: ext counts per depth, shadow counts per depth, scratch
  int *key_hist;      // material-key histogram / offsets [kMaxKeys * 2]
  int *tag;           // regenerating loop: path depth | pass offset << 16, per slot
  WaveLoop *loop;     // regenerating loop state
  int capacity;
  // batch loop only (nullptr otherwise): the batch slot (scene view) of each
  // path slot and of each shadow query
  int *view = nullptr;
  int *sq_view = nullptr;
};
constexpr int kMaxKeys = 256;

// capacity: paths per chunk of the frame (0 = the whole frame); w holds at least that many slots
cudaError_t launch_wave_pass(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                             const WaveBuffers &w, uint32_t *err, int grid, int block, int sort_keys,
                             cudaStream_t st, int trace_budget, int capacity = 0);

// npass passes from pass0 / band0 (band wrapping mod B) over `capacity` path
// slots (<= w.capacity) with path regeneration, as a CUDA-graph while-loop.
// *graph caches the captured loop (rebuilt when a captured argument changes).
struct WaveLoopGraph;
// host_driven: launch the iterations from the host instead (one stream sync each)
cudaError_t launch_wave_loop(const DevScene &s, const DevConfig &c, uint32_t pass0, int band0, int npass, Film f,
                             const WaveBuffers &w, uint32_t *err, int grid, int block, cudaStream_t st,
                             int trace_budget, int capacity, WaveLoopGraph **graph, bool host_driven = false,
                             int limit_override = 0);
void free_wave_loop(WaveLoopGraph *graph);

// ---- path-replay adjoint (adjoint.cu) -----------------------------------------
constexpr int kAdjSharedMax = 4096;  // material-table gradients kept in shared memory (FP64, 32 KB)
int adjoint_shared_params(int pmat);
// adds d(sum of adj-weighted deposits of the pass)/d(params) into grad [M*6*B + E*B*B]
// weight: [npass * W * H] float scratch (each path's adjoint-weighted total); counter: 2 ints
constexpr int kAdjMaxPathsPerLaunch = 1 << 24;  // bounds the weight scratch at 64 MB
cudaError_t launch_adjoint(const DevScene &s, const DevConfig &c, uint32_t pass, int band, const double *adj,
                           double *grad, float *weight, int *counter, uint32_t *err, int grid, cudaStream_t st,
                           int npass = 1, const float *rec = nullptr);
// repack material [M][6][B] and/or EEM [E][B][B] tables given as device arrays
cudaError_t launch_update_materials(float4 *mat, const float *mat_f32, int M, int B, float *eem, float *qy,
                                    float *cdf, const float *eem_src, int E, cudaStream_t st);

// Allocation-free tile pass (render_wave.cu): scratch from a static device array.
int noalloc_max_paths();
size_t noalloc_scratch_bytes();
cudaError_t noalloc_setup(int device, void **ptr);
cudaError_t launch_wave_tile_noalloc(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                                     void *scratch, int x0, int y0, int tw, int th, uint32_t *err, int grid,
                                     int block, cudaStream_t st, int trace_budget);

}  // namespace ts
