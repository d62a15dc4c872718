// One path vertex of the plain megakernel, shared by the single-scene
// megakernel (render_mega.cu) and the multi-scene batch kernel
// (render_batch.cu).
//
// A lane owns one path of cast_rays (main.py:1502-1590) and advances it one
// loop iteration per call: the extension trace of scatter_volume, the
// volume/surface event, next-event estimation with its shadow chain and the
// surface scatter.  Deposits of the path are summed in FP64 and written to the
// film when the path ends or changes band.  With one pass per launch a film
// cell has one owner lane and a plain read-modify-write suffices; a launch of
// several passes shares cells -- volume fluorescence moves a path's deposits
// to another band, i.e. into the plane of another pass of the launch -- so it
// flushes with FP64 atomics (shared = true).
#pragma once
#include "estimator.cuh"
#include "kernels.cuh"

namespace ts {

struct MegaLane {
  PathState p;
  Rng rng;
  int pix;     // pixel of the current path (-1: idle)
  int band;    // the pass's band (transport band)
  int k;       // loop iteration
  double dep;  // pending deposit into p.active_px
  int item;    // work item of the launch (index of its path record)
  bool moved;  // volume fluorescence moved the path to another band
};

// work counters of the counting variant (algorithmic bytes of the roofline)
struct MegaCounts {
  TraceCount tc;
  uint32_t paths = 0, vert = 0, trace = 0, hit = 0, dep = 0;
};

__device__ __forceinline__ void mega_flush(const Film &f, int pixel, int band, double dep, bool shared) {
  if (dep != 0.0 || dep != dep) {
    double *cell = f.block + (size_t)band * f.W * f.H + pixel;
    if (shared) atomicAdd(cell, dep);
    else *cell += dep;  // one owner lane per pixel, band and launch
  }
}

__device__ __forceinline__ void mega_start(const DevScene &s, const DevConfig &c, MegaLane &L, uint32_t pass,
                                           int band, int pixel, int item = 0) {
  L.pix = pixel;
  L.item = item;
  L.moved = false;
  L.band = band;
  L.rng.init(c.seed, pass, (uint32_t)pixel, c.scene_id);
  camera_ray(s, c, pixel % c.W, pixel / c.W, L.rng, L.p, band);
  L.k = 0;
  L.dep = 0.0;
}

// Returns true when the path has ended (its deposit flushed).
template <int W, bool kCount>
__device__ __forceinline__ bool mega_vertex(const DevScene &s, const DevConfig &c, const Film &f, MegaLane &L,
                                            uint32_t &errbits, MegaCounts &cnt, bool shared) {
  PathState &p = L.p;
  const int band = L.band;
  bool done = false;
  // hits beyond ESCAPE count as escapes (main.py:1209-1214): traverse no further
  const Hit h = trace_closest<W, kCount>(s, p.pos, p.dir, c.eps, errbits, &cnt.tc, c.escape);
  const VolEvent ev = volume_event(s, c, p, h, L.rng);
  if (kCount) {
    cnt.trace++;
    cnt.hit += h.slot >= 0;
  }
  if (ev.travel < 0.f) {
    done = true;  // escaped
  } else {
    if (kCount) cnt.vert++;
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
        nee = nee_setup(s, c, p, band, ev.snormal, ev.hit_mat, L.rng, q);
      }
    } else {
      nee = nee_setup(s, c, p, band, ev.snormal, -1, L.rng, q);
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
            trace_closest<W, kCount>(s, ss.pos, q.dir, c.eps, errbits, &cnt.tc, shadow_bound(s, c, q, ss, p.active));
        if (kCount) {
          cnt.trace++;
          cnt.hit += sh.slot >= 0 && sh.slot != q.light_slot;
        }
        if (shadow_segment(s, c, q, sh, p.active, ss)) break;
      }
      if (ss.total > 1e-6f) direct = q.contrib * ss.total;
    }
    if (ev.action == 1 && !done) {
      p.plen++;
      const SurfEvent se = scatter_surface(s, c, p, ev, L.rng);
      apply_surface(c, p, ev, se);
    } else if (ev.action == 2) {
      p.dir = ev.dir;
      p.plen++;
    } else if (ev.action == 3) {
      p.dir = ev.dir;
      if (kCount) cnt.dep += L.dep != 0.0;
      mega_flush(f, L.pix, p.active_px, L.dep, shared);
      L.dep = 0.0;
      L.moved = true;
      p.active = ev.new_wl;
      p.active_px = ev.new_wl;
      p.plen++;
    }
    L.dep += (double)indirect;
    L.dep += (double)direct;
    // A path whose throughput is exactly zero deposits exact zeros from
    // here on (every later term is a product with it), so it ends early.
    if (++L.k >= c.max_depth || p.thr == 0.f) done = true;
  }
  if (done) {
    if (kCount) cnt.dep += L.dep != 0.0;
    mega_flush(f, L.pix, p.active_px, L.dep, shared);
    // the adjoint's replay 0 reads a recorded total instead of re-tracing the path
    if (f.rec) f.rec[L.item] = L.moved ? -1.0f : (float)L.dep;
    L.pix = -1;
  }
  return done;
}

}  // namespace ts
