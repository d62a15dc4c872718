// Plain single-scene renderer: one persistent megakernel per sample pass.
//
// Each lane owns one path (one pixel of cast_rays, main.py:1502-1590) and
// advances it one path vertex per loop iteration: the extension trace of
// scatter_volume, the volume/surface event, next-event estimation with its
// shadow chain, and the surface scatter.  Lanes whose path has ended fetch the
// next pixel with one warp-aggregated atomic, so a warp stays full until the
// pixel pool is exhausted (path regeneration) instead of idling behind its
// longest path.
#include "estimator.cuh"
#include "kernels.cuh"

namespace ts {

namespace {

__device__ __forceinline__ void flush(Film f, int pixel, int band, double dep) {
  if (dep != 0.0 || dep != dep) {
    double *cell = f.block + (size_t)band * f.W * f.H + pixel;
    *cell += dep;  // one owner lane per pixel and pass
  }
}

// kCount: also count the work (for the roofline's algorithmic bytes):
// work[0..7] = paths, path vertices, traversals, node visits, triangle tests,
// surface hits resolved, film deposits, (unused).
template <int W, bool kCount>
__global__ void __launch_bounds__(128, 5) k_render_mega(DevScene s, DevConfig c, uint32_t pass, int band, Film f,
                                                     int *__restrict__ counter, uint32_t *__restrict__ err,
                                                     unsigned long long *__restrict__ work) {
  const int lane = threadIdx.x & 31;
  TraceCount tc;
  uint32_t n_paths = 0, n_vert = 0, n_trace = 0, n_hit = 0, n_dep = 0;
  const int npix = c.W * c.H;
  uint32_t errbits = 0;
  int pix = -1;
  bool exhausted = false;
  PathState p;
  Rng rng;
  int k = 0;
  double dep = 0.0;
  for (;;) {
    const bool need = pix < 0 && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const int idx = base + __popc(m & ((1u << lane) - 1u));
        if (idx < npix) {
          pix = idx;
          if (kCount) n_paths++;
          rng.init(c.seed, pass, (uint32_t)idx, c.scene_id);
          camera_ray(s, c, idx % c.W, idx / c.W, rng, p, band);
          k = 0;
          dep = 0.0;
        } else {
          exhausted = true;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, pix >= 0) == 0) break;
    if (pix < 0) continue;

    // ---- one path vertex (one iteration of the loop at main.py:1534)
    bool done = false;
    // hits beyond ESCAPE count as escapes (main.py:1209-1214): traverse no further
    const Hit h = trace_closest<W, kCount>(s, p.pos, p.dir, c.eps, errbits, &tc, c.escape);
    const VolEvent ev = volume_event(s, c, p, h, rng);
    if (kCount) {
      n_trace++;
      n_hit += h.slot >= 0;
    }
    if (ev.travel < 0.f) {
      done = true;  // escaped
    } else {
      if (kCount) n_vert++;
      p.pos = p.pos + p.dir * ev.travel;
      p.thr *= ev.est;
      float indirect = 0.f, direct = 0.f;
      bool nee = false;
      ShadowQuery q;
      if (ev.action == 1) {
        const Mat sm = get_mat(s, c.B, ev.hit_mat, band);
        if (sm.surf_emis) {
          indirect = emitter_hit(s, c, p, ev, sm.emission);
          done = true;
        } else {
          nee = nee_setup(s, c, p, band, ev.snormal, ev.hit_mat, rng, q);
        }
      } else {
        nee = nee_setup(s, c, p, band, ev.snormal, -1, rng, q);
      }
      if (nee) {
        ShadowState ss;
        ss.pos = q.origin;
        ss.total = 1.f;
        ss.traveled = 0.f;
        ss.vol = q.vol;
        ss.seg = 0;
        for (;;) {
          const Hit sh =
              trace_closest<W, kCount>(s, ss.pos, q.dir, c.eps, errbits, &tc, shadow_bound(s, c, q, ss, p.active));
          if (kCount) {
            n_trace++;
            n_hit += sh.slot >= 0 && sh.slot != q.light_slot;
          }
          if (shadow_segment(s, c, q, sh, p.active, ss)) break;
        }
        if (ss.total > 1e-6f) direct = q.contrib * ss.total;
      }
      if (ev.action == 1 && !done) {
        p.plen++;
        const SurfEvent se = scatter_surface(s, c, p, ev, rng);
        apply_surface(c, p, ev, se);
      } else if (ev.action == 2) {
        p.dir = ev.dir;
        p.plen++;
      } else if (ev.action == 3) {
        p.dir = ev.dir;
        if (kCount) n_dep += dep != 0.0;
        flush(f, pix, p.active_px, dep);
        dep = 0.0;
        p.active = ev.new_wl;
        p.active_px = ev.new_wl;
        p.plen++;
      }
      dep += (double)indirect;
      dep += (double)direct;
      // A path whose throughput is exactly zero deposits exact zeros from
      // here on (every later term is a product with it), so it ends early.
      if (++k >= c.max_depth || p.thr == 0.f) done = true;
    }
    if (done) {
      if (kCount) n_dep += dep != 0.0;
      flush(f, pix, p.active_px, dep);
      pix = -1;
    }
  }
  if (errbits) atomicOr(err, errbits);
  if (kCount) {
    atomicAdd(work + 0, (unsigned long long)n_paths);
    atomicAdd(work + 1, (unsigned long long)n_vert);
    atomicAdd(work + 2, (unsigned long long)n_trace);
    atomicAdd(work + 3, (unsigned long long)tc.nodes);
    atomicAdd(work + 4, (unsigned long long)tc.tris);
    atomicAdd(work + 5, (unsigned long long)n_hit);
    atomicAdd(work + 6, (unsigned long long)n_dep);
  }
}

}  // namespace

cudaError_t launch_render_mega(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                               int *counter, uint32_t *err, int grid, int block, cudaStream_t st,
                               unsigned long long *work) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  block = block > 128 ? 128 : block;  // the kernel is compiled for blocks of at most 128 threads
  if (s.node_width == 8) {
    if (work) k_render_mega<8, true><<<grid, block, 0, st>>>(s, c, pass, band, f, counter, err, work);
    else k_render_mega<8, false><<<grid, block, 0, st>>>(s, c, pass, band, f, counter, err, nullptr);
  } else if (s.node_width == 4) {
    if (work) k_render_mega<4, true><<<grid, block, 0, st>>>(s, c, pass, band, f, counter, err, work);
    else k_render_mega<4, false><<<grid, block, 0, st>>>(s, c, pass, band, f, counter, err, nullptr);
  } else if (c.speculative) {
    if (work) k_render_mega<3, true><<<grid, block, 0, st>>>(s, c, pass, band, f, counter, err, work);
    else k_render_mega<3, false><<<grid, block, 0, st>>>(s, c, pass, band, f, counter, err, nullptr);
  } else {
    if (work) k_render_mega<2, true><<<grid, block, 0, st>>>(s, c, pass, band, f, counter, err, work);
    else k_render_mega<2, false><<<grid, block, 0, st>>>(s, c, pass, band, f, counter, err, nullptr);
  }
  return cudaGetLastError();
}

}  // namespace ts
