// Wavefront renderer: one sample pass as a fixed sequence of stage kernels
// joined by compacted queues in device memory.
//
//   generate            camera rays for every pixel -> extension queue Q0
//   trace(k)            closest hit for every path in Qk, and the whole shadow
//                       chain (<= scatter_bounces segments) of every query
//                       left by shade(k-1); direct light is deposited here
//   shade(k)            volume event, emitter hit, next-event setup and surface
//                       scatter for every path of Qk -> Q(k+1), shadow queries
//   trace(depth)        the last shadow queries
//
// Path state lives in SoA arrays indexed by pixel; queues hold pixel ids.
// Every stage fetches work 32 items at a time with one atomic per warp, so
// the grid is persistent (a multiple of the SM count) and independent of
// queue lengths, which are only known on the device.  Each pixel owns one
// path per pass and stages run in stream order, so film deposits need no
// atomics.  With sort_keys set, the shading queue is reordered by the hit
// material (a counting sort on the device) so that warps shade one material
// at a time.
#include <cstring>
#include <mutex>
#include <vector>

#include "batch.cuh"
#include "estimator.cuh"
#include "kernels.cuh"

namespace ts {

namespace {

// layout of WaveBuffers::counts
constexpr int kMaxDepth = 1024;
constexpr int kCntExt = 0;                      // [kMaxDepth+1] extension queue lengths
constexpr int kCntSh = kCntExt + kMaxDepth + 1;  // [kMaxDepth+1] shadow queue lengths
constexpr int kCntFetchT = kCntSh + kMaxDepth + 1;
constexpr int kCntFetchS = kCntFetchT + kMaxDepth + 1;
constexpr int kCntTotal = kCntFetchS + kMaxDepth + 1;

__device__ __forceinline__ int warp_fetch(int *ctr) {
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0) base = atomicAdd(ctr, 32);
  return __shfl_sync(0xffffffffu, base, 0);
}

// append with one atomic per warp; returns the slot for lanes with want=true
__device__ __forceinline__ int warp_append(int *ctr, bool want) {
  const unsigned m = __ballot_sync(0xffffffffu, want);
  if (!m) return -1;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(ctr, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  return want ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

// shared: several passes in flight may deposit into one cell (fluorescence
// moves a deposit into another pass's band), so the add is atomic
__device__ __forceinline__ void deposit(const Film &f, int pixel, int band, float v, bool shared = false) {
  if (v == 0.f) return;
  double *cell = f.block + (size_t)band * f.W * f.H + pixel;
  if (shared) atomicAdd(cell, (double)v);
  else *cell += (double)v;
}

// the camera ray of one pixel into path slot `slot` (the pixel id keys the random stream)
__device__ __forceinline__ void start_path(float3 o, float3 cu, float3 cv, float3 cw, const DevConfig &c,
                                           uint32_t pass, int band, int pix, const WaveBuffers &w, int slot) {
  Rng rng;
  rng.init(c.seed, pass, (uint32_t)pix, c.scene_id);
  PathState ps;
  camera_ray(o, cu, cv, cw, c, pix % c.W, pix / c.W, rng, ps, band);
  w.pos_thr[slot] = make_float4(ps.pos.x, ps.pos.y, ps.pos.z, ps.thr);
  w.dir_spdf[slot] = make_float4(ps.dir.x, ps.dir.y, ps.dir.z, ps.spdf);
  w.meta[slot] = make_int4(pix, band | (band << 8), 0, (int)rng.n);
}

// camera rays of pixels [p0, p0 + n): path slot q <-> pixel p0 + q
__global__ void k_generate(DevScene s, DevConfig c, uint32_t pass, int band, WaveBuffers w, int p0, int n) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    start_path(s.cam_o, s.cam_u, s.cam_v, s.cam_w, c, pass, band, p0 + q, w, q);
    w.queue[0][q] = q;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) w.counts[kCntExt + 0] = n;
}

// trace(k): shadow chains of shade(k-1), then extension hits of Qk.
// Persistent lanes with per-lane refill: each lane traverses its current ray
// for at most `budget` steps; lanes whose ray has finished then take new work
// items (one atomic per warp), so a warp does not idle behind its longest ray.
// kLoop: one iteration of the regenerating loop (queue lengths from *L).
template <int W, bool kLoop = false>
__global__ void __launch_bounds__(kMaxBlock, 4) k_trace(DevScene s, DevConfig c, int depth, Film f, WaveBuffers w,
                                                     uint32_t *__restrict__ err, int budget, int ext_sorted,
                                                     int shadow_sorted, WaveLoop *L) {
  uint32_t eb = 0;
  int nsh, next, *fetch;
  const int *q;
  bool shared = false;
  if (kLoop) {
    const int a = L->iter & 1;
    nsh = L->sh[a ^ 1];
    next = L->ext[a];
    q = w.queue[a];
    fetch = L->fetch + 0;
    shared = L->shared != 0;
    ext_sorted = shadow_sorted = 0;
  } else {
    nsh = depth > 0 ? w.counts[kCntSh + depth - 1] : 0;
    next = depth < c.max_depth ? w.counts[kCntExt + depth] : 0;
    q = ext_sorted ? w.trace_order : w.queue[depth & 1];
    fetch = w.counts + kCntFetchT + depth;
  }
  const int total = nsh + next;
  const int lane = threadIdx.x & 31;
  int item = -1, pid = 0, pixel = 0, band = 0, dep_band = 0;
  bool exhausted = false;
  Traversal t;
  int2 stack[StackSize<W>::value];
#ifdef TS_SHORT_STACK
  // measurement variant: the newest TS_SHORT_STACK entries of each lane's
  // wide-node stack in shared memory (dynamic, TS_SHORT_STACK x block entries)
  extern __shared__ int2 short_stack_smem[];
  ShortStack<TS_SHORT_STACK> sst{short_stack_smem, stack, (int)blockDim.x, (int)threadIdx.x, 0};
#endif
  ShadowQuery sq;
  ShadowState ss;
  for (;;) {
    const bool need = item < 0 && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(fetch, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const int idx = base + __popc(m & ((1u << lane) - 1u));
        if (idx >= total) {
          exhausted = true;
        } else if (idx < nsh) {
          item = idx;
          const int qi = shadow_sorted ? w.shadow_order[idx] : idx;
          const float4 o = w.sq_origin[qi], d = w.sq_dir[qi];
          const int4 mm = w.sq_meta[qi];
          sq.origin = xyz(o);
          sq.max_dist = o.w;
          sq.dir = xyz(d);
          sq.contrib = d.w;
          sq.light_slot = mm.y;
          sq.vol = mm.z;
          pixel = mm.x;
          band = mm.w & 0xff;
          dep_band = mm.w >> 8;
          ss.pos = sq.origin;
          ss.total = 1.f;
          ss.traveled = 0.f;
          ss.vol = sq.vol;
          ss.seg = 0;
          trav_begin(s, t, ss.pos, sq.dir, shadow_bound(s, c, sq, ss, band));
        } else {
          item = idx;
          pid = q[idx - nsh];
          const float4 pt = w.pos_thr[pid], ds = w.dir_spdf[pid];
          trav_begin(s, t, xyz(pt), xyz(ds), c.escape);
        }
      }
    }
    if (__ballot_sync(0xffffffffu, item >= 0) == 0) break;
    bool done = false;
#if defined(TS_IDLE_REFILL)
    // measurement variant: the warp steps its rays one traversal step at a
    // time and refills as soon as TS_IDLE_REFILL lanes could take new work
    // (dynamic fetch), within the same bound of `budget` steps
    for (int st = 0; st < budget; ++st) {
      if (item >= 0 && !done) done = trav_advance<W>(s, t, stack, c.eps, 1, eb);
      if (__popc(__ballot_sync(0xffffffffu, done || (item < 0 && !exhausted))) >= TS_IDLE_REFILL) break;
    }
#else
    if (item >= 0) {
#ifdef TS_SHORT_STACK
      if constexpr (W == 4 || W == 8) done = trav_steps_wide<W>(s, t, sst, c.eps, budget, eb);
      else done = trav_advance<W>(s, t, stack, c.eps, budget, eb);
#else
      done = trav_advance<W>(s, t, stack, c.eps, budget, eb);
#endif
    }
#endif
    if (done) {
      if (item < nsh) {
        if (shadow_segment(s, c, sq, t.h, band, ss)) {
          if (ss.total > 1e-6f) deposit(f, pixel, dep_band, sq.contrib * ss.total, shared);
          item = -1;
        } else {
          trav_begin(s, t, ss.pos, sq.dir, shadow_bound(s, c, sq, ss, band));
        }
      } else {
        w.hit[pid] = make_float4(t.h.t, t.h.u, t.h.v, __int_as_float(t.h.slot));
        item = -1;
      }
    }
  }
  if (eb) atomicOr(err, eb);
}

template <bool kLoop = false>
void launch_trace(const DevScene &s, const DevConfig &c, int depth, Film f, const WaveBuffers &w, uint32_t *err,
                  int grid, int block, cudaStream_t st, int budget, int ext_sorted = 0, int shadow_sorted = 0,
                  WaveLoop *L = nullptr) {
#ifdef TS_SHORT_STACK
  const size_t smem = (size_t)TS_SHORT_STACK * block * sizeof(int2);
#else
  const size_t smem = 0;
#endif
  if (s.node_width == 9)
    k_trace<9, kLoop><<<grid, block, smem, st>>>(s, c, depth, f, w, err, budget, ext_sorted, shadow_sorted, L);
  else if (s.node_width == 5)
    k_trace<5, kLoop><<<grid, block, smem, st>>>(s, c, depth, f, w, err, budget, ext_sorted, shadow_sorted, L);
  else if (s.node_width == 8)
    k_trace<8, kLoop><<<grid, block, smem, st>>>(s, c, depth, f, w, err, budget, ext_sorted, shadow_sorted, L);
  else if (s.node_width == 4)
    k_trace<4, kLoop><<<grid, block, smem, st>>>(s, c, depth, f, w, err, budget, ext_sorted, shadow_sorted, L);
  else if (c.speculative)
    k_trace<3, kLoop><<<grid, block, smem, st>>>(s, c, depth, f, w, err, budget, ext_sorted, shadow_sorted, L);
  else
    k_trace<2, kLoop><<<grid, block, smem, st>>>(s, c, depth, f, w, err, budget, ext_sorted, shadow_sorted, L);
}

// ---- queue sorting ------------------------------------------------------
// Counting sorts that reorder a queue by a small key so that neighbouring
// lanes of a warp take similar work: the shading queue by (hit material,
// medium the path travels in) -- by material alone when the pairs outnumber
// the key table --, the extension rays by direction octant, the shadow queries
// by light triangle.
// Each is count (block histograms) -> scan -> scatter (one atomic per key per
// warp, lanes of equal keys grouped with __match_any_sync).
enum SortKind { kSortShade = 0, kSortExt = 1, kSortShadow = 2 };
constexpr int kExtKeys = 8, kShadowKeys = 16;

__device__ __forceinline__ int sort_count_of(const WaveBuffers &w, int kind, int depth) {
  return kind == kSortShadow ? w.counts[kCntSh + depth] : w.counts[kCntExt + depth];
}

__device__ __forceinline__ int sort_item(const WaveBuffers &w, int kind, int depth, int i) {
  return kind == kSortShadow ? i : w.queue[depth & 1][i];
}

__device__ __forceinline__ int sort_key(const DevScene &s, const WaveBuffers &w, int kind, int item, int nkeys) {
  int key;
  if (kind == kSortShade) {
    const int M = s.num_materials;
    const int slot = __float_as_int(w.hit[item].w);
    key = slot >= 0 ? __float_as_int(__ldg(s.tri + 3 * (size_t)slot + 1).w) : M;
    if ((M + 1) * M <= nkeys) key = key * M + w.meta[item].z;  // (material, medium)
  } else if (kind == kSortExt) {
    const float4 d = w.dir_spdf[item];
    key = (d.x < 0.f ? 1 : 0) | (d.y < 0.f ? 2 : 0) | (d.z < 0.f ? 4 : 0);
  } else {
    key = w.sq_meta[item].y;
  }
  return kind == kSortShade ? (key < nkeys ? key : nkeys - 1) : (key & (nkeys - 1));
}

__global__ void k_sort_count(DevScene s, int depth, WaveBuffers w, int kind, int nkeys) {
  __shared__ int hist[kMaxKeys];
  for (int k = threadIdx.x; k < nkeys; k += blockDim.x) hist[k] = 0;
  __syncthreads();
  const int n = sort_count_of(w, kind, depth);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(&hist[sort_key(s, w, kind, sort_item(w, kind, depth, i), nkeys)], 1);
  __syncthreads();
  for (int k = threadIdx.x; k < nkeys; k += blockDim.x)
    if (hist[k]) atomicAdd(&w.key_hist[k], hist[k]);
}

__global__ void k_sort_scan(WaveBuffers w, int nkeys) {
  if (threadIdx.x == 0) {
    int run = 0;
    for (int k = 0; k < nkeys; ++k) {
      const int v = w.key_hist[k];
      w.key_hist[kMaxKeys + k] = run;  // running insert position
      w.key_hist[k] = 0;               // cleared for the next sort
      run += v;
    }
  }
}

__global__ void k_sort_scatter(DevScene s, int depth, WaveBuffers w, int kind, int nkeys, int *__restrict__ out) {
  const int n = sort_count_of(w, kind, depth);
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
    const int i = base + lane;
    const bool valid = i < n;
    const unsigned active = __ballot_sync(0xffffffffu, valid);
    if (!valid) continue;
    const int item = sort_item(w, kind, depth, i);
    const int key = sort_key(s, w, kind, item, nkeys);
    const unsigned peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    int pos = 0;
    if (lane == leader) pos = atomicAdd(&w.key_hist[kMaxKeys + key], __popc(peers));
    pos = __shfl_sync(peers, pos, leader);
    out[pos + __popc(peers & ((1u << lane) - 1u))] = item;
  }
}

void launch_sort(const DevScene &s, int depth, const WaveBuffers &w, int kind, int nkeys, int *out, int grid,
                 cudaStream_t st) {
  k_sort_count<<<grid, 256, 0, st>>>(s, depth, w, kind, nkeys);
  k_sort_scan<<<1, 32, 0, st>>>(w, nkeys);
  k_sort_scatter<<<grid, 256, 0, st>>>(s, depth, w, kind, nkeys, out);
}

// one path of an extension queue: volume event, emitter hit, next-event setup
// and surface or volume scatter.  cont: the path goes on (its state was
// written back); nee: r.sq is its shadow query.  last: no further vertex.
struct Shaded {
  bool cont, nee;
  int pix, dep_band;
  ShadowQuery sq;
};

__device__ __forceinline__ void shade_path(const DevScene &s, const DevConfig &c, uint32_t pass, int band, bool last,
                                           const Film &f, const WaveBuffers &w, int pid, bool shared, Shaded &r) {
  const float4 pt = w.pos_thr[pid], ds = w.dir_spdf[pid];
  const int4 m = w.meta[pid];
  const float4 hh = w.hit[pid];
  r.pix = m.x;
  PathState p;
  p.pos = xyz(pt);
  p.thr = pt.w;
  p.dir = xyz(ds);
  p.spdf = ds.w;
  p.active = m.y & 0xff;
  p.active_px = (m.y >> 8) & 0xff;
  p.plen = (m.y >> 16) & 0xffff;
  p.vol = m.z;
  Rng rng;
  rng.init(c.seed, pass, (uint32_t)m.x, c.scene_id, (uint32_t)m.w);
  Hit h;
  h.t = hh.x;
  h.u = hh.y;
  h.v = hh.z;
  h.slot = __float_as_int(hh.w);
  const VolEvent ev = volume_event(s, c, p, h, rng);
  if (ev.travel < 0.f) return;
  p.pos = p.pos + p.dir * ev.travel;
  p.thr *= ev.est;
  bool done = false;
  float indirect = 0.f;
  if (ev.action == 1) {
    const Mat sm = get_mat(s, c.B, ev.hit_mat, band);
    if (sm.surf_emis) {
      indirect = emitter_hit(s, c, p, ev, sm.emission);
      done = true;
    } else {
      r.nee = nee_setup(s, c, p, band, ev.snormal, ev.hit_mat, rng, r.sq);
    }
  } else {
    r.nee = nee_setup(s, c, p, band, ev.snormal, -1, rng, r.sq);
  }
  r.sq.band = p.active;
  if (ev.action == 1 && !done) {
    p.plen++;
    const SurfEvent se = scatter_surface(s, c, p, ev, rng);
    apply_surface(c, p, ev, se);
  } else if (ev.action == 2) {
    p.dir = ev.dir;
    p.plen++;
  } else if (ev.action == 3) {
    p.dir = ev.dir;
    p.active = ev.new_wl;
    p.active_px = ev.new_wl;
    p.plen++;
  }
  r.dep_band = p.active_px;
  deposit(f, m.x, r.dep_band, indirect, shared);
  r.cont = !done && !last && p.thr != 0.f;
  if (r.cont) {
    w.pos_thr[pid] = make_float4(p.pos.x, p.pos.y, p.pos.z, p.thr);
    w.dir_spdf[pid] = make_float4(p.dir.x, p.dir.y, p.dir.z, p.spdf);
    w.meta[pid] = make_int4(m.x, p.active | (p.active_px << 8) | (p.plen << 16), p.vol, (int)rng.n);
  }
}

// Queue appends are bounded by construction (every slot appends at most once
// per stage); the checks below only keep a corrupted counter from writing
// past a queue, reporting kErrQueueOverflow instead.
__device__ __forceinline__ void append_shadow(int *count, const WaveBuffers &w, const Shaded &r, uint32_t *err,
                                              int view = -1) {
  const int sslot = warp_append(count, r.nee);
  if (r.nee && sslot >= w.capacity) {
    atomicOr(err, kErrQueueOverflow);
    return;
  }
  if (r.nee) {
    if (w.sq_view) w.sq_view[sslot] = view;
    w.sq_origin[sslot] = make_float4(r.sq.origin.x, r.sq.origin.y, r.sq.origin.z, r.sq.max_dist);
    w.sq_dir[sslot] = make_float4(r.sq.dir.x, r.sq.dir.y, r.sq.dir.z, r.sq.contrib);
    w.sq_meta[sslot] = make_int4(r.pix, r.sq.light_slot, r.sq.vol, r.sq.band | (r.dep_band << 8));
  }
}

__device__ __forceinline__ void append_ext(int *count, int *q, int pid, bool want, int capacity, uint32_t *err) {
  const int slot = warp_append(count, want);
  if (!want) return;
  if (slot < capacity) q[slot] = pid;
  else atomicOr(err, kErrQueueOverflow);
}

__global__ void __launch_bounds__(kMaxBlock) k_shade(DevScene s, DevConfig c, uint32_t pass, int band, int depth,
                                               Film f, WaveBuffers w, int use_sorted, uint32_t *err) {
  const int n = w.counts[kCntExt + depth];
  const int *q = use_sorted ? w.sorted : w.queue[depth & 1];
  int *qn = w.queue[(depth + 1) & 1];
  int *fetch = w.counts + kCntFetchS + depth;
  const bool last = depth + 1 >= c.max_depth;
  for (;;) {
    const int base = warp_fetch(fetch);
    if (base >= n) break;
    const int i = base + (threadIdx.x & 31);
    Shaded r;
    r.cont = r.nee = false;
    r.pix = -1;
    r.dep_band = 0;
    int pid = -1;
    if (i < n) {
      pid = q[i];
      shade_path(s, c, pass, band, last, f, w, pid, false, r);
    }
    append_shadow(w.counts + kCntSh + depth, w, r, err);
    append_ext(w.counts + kCntExt + depth + 1, qn, pid, r.cont, w.capacity, err);
  }
}

// ---- the regenerating loop ----------------------------------------------
// A launch of npass passes (a wavelength bundle, or one pass) as work items
// idx = pass offset * npix + pixel over `capacity` path slots.  One iteration
// is trace (the shadow queries of the last shade and the extension rays of
// the queue) then shade, in which every slot whose path has ended starts the
// next work item at once, so the queue stays full until the items run out
// and the long-path tail is paid once per launch, not once per pass.  The
// iterations run as the body of a CUDA-graph while-loop whose condition the
// control kernel sets: no host round trip decides when a launch is done.
//
// Slot tag: path depth | pass offset << 16.  Each cell of a pass's band plane
// has one path per pass, so deposits are plain adds unless passes in flight
// share cells (several passes with fluorescence moving deposits across bands).

// paths [0, n0) of the launch into slots [0, n0), and the loop state
__global__ void k_loop_init(DevScene s, DevConfig c, WaveBuffers w, WaveLoop *L, uint32_t pass0, int band0,
                            int npass, int n0, int limit, int shared) {
  const int npix = c.W * c.H;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n0; q += gridDim.x * blockDim.x) {
    const int po = q / npix;
    int band = band0 + po;
    if (band >= c.B) band -= c.B;
    start_path(s.cam_o, s.cam_u, s.cam_v, s.cam_w, c, pass0 + (uint32_t)po, band, q - po * npix, w, q);
    w.tag[q] = po << 16;
    w.queue[0][q] = q;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    L->ext[0] = n0;
    L->ext[1] = 0;
    L->sh[0] = L->sh[1] = 0;
    L->fetch[0] = L->fetch[1] = 0;
    L->next_item = n0;
    L->total = npass * npix;
    L->iter = 0;
    L->limit = limit;
    L->pass0 = pass0;
    L->band0 = band0;
    L->shared = shared;
    L->cam_o = s.cam_o;
    L->cam_u = s.cam_u;
    L->cam_v = s.cam_v;
    L->cam_w = s.cam_w;
  }
}

// 64 registers (4 resident 256-thread blocks per SM; a few spills): faster
// than the unbounded 111-register build by 4-6 % on whole-bundle loops
__global__ void __launch_bounds__(kMaxBlock, 4) k_shade_loop(DevScene s, DevConfig c, Film f, WaveBuffers w, WaveLoop *L,
                                                          uint32_t *err) {
  const int a = L->iter & 1;
  const int n = L->ext[a];
  const int *q = w.queue[a];
  int *qn = w.queue[a ^ 1];
  const uint32_t pass0 = L->pass0;
  const int band0 = L->band0, total = L->total;
  const bool shared = L->shared != 0;
  // items left to start, read once: the item counter then overshoots the
  // total by at most one claim per slot
  const bool more = L->next_item < total;
  const int npix = c.W * c.H;
  for (;;) {
    const int base = warp_fetch(L->fetch + 1);
    if (base >= n) break;
    const int i = base + (threadIdx.x & 31);
    Shaded r;
    r.cont = r.nee = false;
    r.pix = -1;
    r.dep_band = 0;
    int pid = -1;
    if (i < n) {
      pid = q[i];
      const int tag = w.tag[pid];
      const int po = tag >> 16;
      int band = band0 + po;
      if (band >= c.B) band -= c.B;
      shade_path(s, c, pass0 + (uint32_t)po, band, (tag & 0xffff) + 1 >= c.max_depth, f, w, pid, shared, r);
      if (r.cont) w.tag[pid] = tag + 1;
    }
    append_shadow(L->sh + a, w, r, err);
    // the slots of ended paths start the next work items
    bool fresh = false;
    if (more) {
      const int item = warp_append(&L->next_item, pid >= 0 && !r.cont);
      if (item >= 0 && item < total) {
        const int po = item / npix;
        int band = band0 + po;
        if (band >= c.B) band -= c.B;
        start_path(L->cam_o, L->cam_u, L->cam_v, L->cam_w, c, pass0 + (uint32_t)po, band, item - po * npix, w, pid);
        w.tag[pid] = po << 16;
        fresh = true;
      }
    }
    append_ext(L->ext + (a ^ 1), qn, pid, r.cont || fresh, w.capacity, err);
  }
}

// end of an iteration: go on while rays or shadow queries are queued, reset
// the counters the next iteration appends to, and stop (with an error bit) at
// the iteration bound, which no launch reaches unless the queues are corrupt
__global__ void k_loop_control(WaveLoop *L, cudaGraphConditionalHandle h, int in_graph, uint32_t *err) {
  if (threadIdx.x != 0) return;
  const int a = L->iter & 1;
  bool go = L->ext[a ^ 1] > 0 || L->sh[a] > 0;
  L->ext[a] = 0;
  L->sh[a ^ 1] = 0;
  L->fetch[0] = L->fetch[1] = 0;
  const int it = L->iter + 1;
  L->iter = it;
  if (go && it >= L->limit) {
    atomicOr(err, kErrIterationCap);
    go = false;
  }
  L->go = go ? 1 : 0;
  if (in_graph) cudaGraphSetConditional(h, go ? 1u : 0u);
}

}  // namespace

cudaError_t launch_wave_chunk(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                              const WaveBuffers &w, uint32_t *err, int grid, int block, int sort_keys,
                              cudaStream_t st, int trace_budget, int p0, int n);

cudaError_t launch_wave_pass(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                             const WaveBuffers &w, uint32_t *err, int grid, int block, int sort_keys,
                             cudaStream_t st, int trace_budget, int capacity) {
  // the frame in chunks of at most `capacity` paths (their queues stay in L2)
  const int npix = c.W * c.H;
  const int chunk = capacity > 0 && capacity < npix ? capacity : npix;
  for (int p0 = 0; p0 < npix; p0 += chunk) {
    const cudaError_t e = launch_wave_chunk(s, c, pass, band, f, w, err, grid, block, sort_keys, st, trace_budget, p0,
                                            npix - p0 < chunk ? npix - p0 : chunk);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_wave_chunk(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                              const WaveBuffers &w, uint32_t *err, int grid, int block, int sort_keys,
                              cudaStream_t st, int trace_budget, int p0, int n) {
  if (c.max_depth > kMaxDepth) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(w.counts, 0, kCntTotal * sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int gen_grid = (n + 255) / 256;
  k_generate<<<gen_grid, 256, 0, st>>>(s, c, pass, band, w, p0, n);
  // sort_keys bit 0: shading queue by material; bit 1: extension rays by
  // direction octant; bit 2: shadow queries by light triangle
  const int M = s.num_materials;
  const int nmat = (M + 1) * M <= kMaxKeys ? (M + 1) * M : (M + 1 < kMaxKeys ? M + 1 : kMaxKeys);
  if (sort_keys) {
    e = cudaMemsetAsync(w.key_hist, 0, 2 * kMaxKeys * sizeof(int), st);
    if (e != cudaSuccess) return e;
  }
  const int sort_grid = grid < 4 * 148 ? grid : 4 * 148;
  for (int d = 0; d < c.max_depth; ++d) {
    const int ext_sorted = (sort_keys & 2) ? 1 : 0;
    const int sh_sorted = (sort_keys & 4) && d > 0 ? 1 : 0;
    if (ext_sorted) launch_sort(s, d, w, kSortExt, kExtKeys, w.trace_order, sort_grid, st);
    if (sh_sorted) launch_sort(s, d - 1, w, kSortShadow, kShadowKeys, w.shadow_order, sort_grid, st);
    launch_trace(s, c, d, f, w, err, grid, block, st, trace_budget, ext_sorted, sh_sorted);
    if (sort_keys & 1) launch_sort(s, d, w, kSortShade, nmat, w.sorted, sort_grid, st);
    k_shade<<<grid, block, 0, st>>>(s, c, pass, band, d, f, w, (sort_keys & 1) ? 1 : 0, err);
  }
  // the last depth's shadow queries
  if (c.max_depth > 0) {
    const int sh_sorted = (sort_keys & 4) ? 1 : 0;
    if (sh_sorted) launch_sort(s, c.max_depth - 1, w, kSortShadow, kShadowKeys, w.shadow_order, sort_grid, st);
    launch_trace(s, c, c.max_depth, f, w, err, grid, block, st, trace_budget, 0, sh_sorted);
  }
  return cudaGetLastError();
}

struct WaveLoopGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t capture = nullptr;
  std::vector<unsigned char> key;  // the captured kernel arguments
};

void free_wave_loop(WaveLoopGraph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->capture) cudaStreamDestroy(g->capture);
  delete g;
}

namespace {

cudaError_t build_wave_loop(WaveLoopGraph &G, const DevScene &s, const DevConfig &c, Film f, const WaveBuffers &w,
                            uint32_t *err, int grid, int block, int budget) {
  if (G.exec) cudaGraphExecDestroy(G.exec);
  if (G.graph) cudaGraphDestroy(G.graph);
  G.exec = nullptr;
  G.graph = nullptr;
  cudaError_t e;
  if (!G.capture && (e = cudaStreamCreateWithFlags(&G.capture, cudaStreamNonBlocking)) != cudaSuccess) return e;
  if ((e = cudaGraphCreate(&G.graph, 0)) != cudaSuccess) return e;
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, G.graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, G.graph, nullptr, 0, &cp)) != cudaSuccess) return e;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(G.capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return e;
  launch_trace<true>(s, c, 0, f, w, err, grid, block, G.capture, budget, 0, 0, w.loop);
  k_shade_loop<<<grid, block, 0, G.capture>>>(s, c, f, w, w.loop, err);
  k_loop_control<<<1, 32, 0, G.capture>>>(w.loop, h, 1, err);
  const cudaError_t le = cudaGetLastError();
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(G.capture, &captured);
  if (le != cudaSuccess) return le;
  if (e != cudaSuccess) return e;
  return cudaGraphInstantiate(&G.exec, G.graph, 0);
}

}  // namespace

cudaError_t launch_wave_loop(const DevScene &s, const DevConfig &c, uint32_t pass0, int band0, int npass, Film f,
                             const WaveBuffers &w, uint32_t *err, int grid, int block, cudaStream_t st,
                             int trace_budget, int capacity, WaveLoopGraph **graph, bool host_driven,
                             int limit_override) {
  const int64_t npix = (int64_t)c.W * c.H;
  const int64_t total = npix * npass;
  if (c.max_depth > kMaxDepth || npass < 1 || npass > 32767 || capacity < 1 || capacity > w.capacity ||
      !w.tag || !w.loop || total + capacity > INT32_MAX)
    return cudaErrorInvalidValue;
  if (c.max_depth <= 0) return cudaSuccess;  // no vertex: nothing is deposited (as in the depth-synchronous pass)
  const int n0 = (int)(total < capacity ? total : capacity);
  // every slot starts a new item at least once per max_depth iterations while
  // items are left, and a path lives at most max_depth iterations
  const int64_t bound = ((total + n0 - 1) / n0 + 2) * (int64_t)(c.max_depth + 1) + 4;
  int limit = (int)(bound < INT32_MAX ? bound : INT32_MAX);
  if (limit_override > 0 && limit_override < limit) limit = limit_override;  // a caller's tighter bound
  const int shared = npass > 1 && s.num_eems > 0 ? 1 : 0;
  struct Key {
    DevScene s;
    DevConfig c;
    Film f;
    WaveBuffers w;
    uint32_t *err;
    int grid, block, budget;
  } k;
  memset(&k, 0, sizeof k);
  memcpy(&k.s, &s, sizeof s);
  // the loop kernels take the camera from the loop state: moving it needs no new graph
  memset(&k.s.cam_o, 0, sizeof k.s.cam_o);
  memset(&k.s.cam_u, 0, sizeof k.s.cam_u);
  memset(&k.s.cam_v, 0, sizeof k.s.cam_v);
  memset(&k.s.cam_w, 0, sizeof k.s.cam_w);
  memcpy(&k.c, &c, sizeof c);
  memcpy(&k.f, &f, sizeof f);
  memcpy(&k.w, &w, sizeof w);
  k.err = err;
  k.grid = grid;
  k.block = block;
  k.budget = trace_budget;
  const unsigned char *kb = reinterpret_cast<const unsigned char *>(&k);
  if (host_driven) {
    const int init_grid = (int)((n0 + 255) / 256 < 4096 ? (n0 + 255) / 256 : 4096);
    k_loop_init<<<init_grid, 256, 0, st>>>(s, c, w, w.loop, pass0, band0, npass, n0, limit, shared);
    for (int it = 0; it < limit; ++it) {
      launch_trace<true>(s, c, 0, f, w, err, grid, block, st, trace_budget, 0, 0, w.loop);
      k_shade_loop<<<grid, block, 0, st>>>(s, c, f, w, w.loop, err);
      k_loop_control<<<1, 32, 0, st>>>(w.loop, 0, 0, err);
      int go = 0;
      cudaError_t e = cudaMemcpyAsync(&go, &w.loop->go, sizeof(int), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return e;
      if (!go) break;
    }
    return cudaGetLastError();
  }
  if (!*graph) *graph = new WaveLoopGraph;
  WaveLoopGraph &G = **graph;
  if (!G.exec || G.key.size() != sizeof k || memcmp(G.key.data(), kb, sizeof k) != 0) {
    G.key.clear();
    const cudaError_t e = build_wave_loop(G, s, c, f, w, err, grid, block, trace_budget);
    if (e != cudaSuccess) return e;
    G.key.assign(kb, kb + sizeof k);
  }
  const int init_grid = (int)((n0 + 255) / 256 < 4096 ? (n0 + 255) / 256 : 4096);
  k_loop_init<<<init_grid, 256, 0, st>>>(s, c, w, w.loop, pass0, band0, npass, n0, limit, shared);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaGraphLaunch(G.exec, st);
}

// ---------------------------------------------------------------------------
// The batch loop: many scene views (batch slots, each a context's scene,
// camera, resolution, depth and film) in one regenerating wavefront loop.
// The work items of a step are the concatenation of the active slots' items
// (a whole spectral block of each, k_batch_prepare); a path slot carries the
// view of its item in w.view and a shadow query in w.sq_view, and every stage
// reads that view's scene, config and film from the slot table.  Paths are
// exactly those of ts_render_pass on each view's context: the same random
// streams (seed, pass, pixel, scene id), the same event functions.
namespace {

// item -> view, pass offset and pixel of the current step
struct BatchItem {
  int view, po, pix;
};
__device__ __forceinline__ BatchItem batch_item(const BatchSlot *slots, int n, int item) {
  BatchItem r;
  r.view = batch_find_slot(slots, n, item);
  const BatchSlot &sl = slots[r.view];
  const int npix = sl.c.W * sl.c.H;
  const int local = item - sl.item0;
  r.po = local / npix;
  r.pix = local - r.po * npix;
  return r;
}

__device__ __forceinline__ int slot_band(const BatchSlot &sl, int po) {
  int b = sl.band0 + po;
  return b >= sl.c.B ? b - sl.c.B : b;
}

// deposits share film cells between passes in flight only where fluorescence moves them
__device__ __forceinline__ bool slot_shared(const BatchSlot &sl) { return sl.s.num_eems > 0; }

__device__ __forceinline__ void start_batch_path(const BatchSlot *slots, int n, const WaveBuffers &w, int item,
                                                 int q) {
  const BatchItem it = batch_item(slots, n, item);
  const BatchSlot &sl = slots[it.view];
  start_path(sl.s.cam_o, sl.s.cam_u, sl.s.cam_v, sl.s.cam_w, sl.c, sl.pass0 + (uint32_t)it.po, slot_band(sl, it.po),
             it.pix, w, q);
  w.tag[q] = it.po << 16;
  w.view[q] = it.view;
}

__global__ void k_bloop_init(const BatchSlot *__restrict__ slots, int n, const BatchHeader *__restrict__ h,
                             WaveBuffers w, WaveLoop *L, int capacity, int limit) {
  const int total = h->total;
  const int n0 = total < capacity ? total : capacity;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n0; q += gridDim.x * blockDim.x) {
    start_batch_path(slots, n, w, q, q);
    w.queue[0][q] = q;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    L->ext[0] = n0;
    L->ext[1] = 0;
    L->sh[0] = L->sh[1] = 0;
    L->fetch[0] = L->fetch[1] = 0;
    L->next_item = n0;
    L->total = total;
    L->iter = 0;
    L->limit = limit;
    L->go = n0 > 0 ? 1 : 0;
  }
}

// trace stage of the batch loop: k_trace<W, true> with each item's view
template <int W>
__global__ void __launch_bounds__(kMaxBlock, 4) k_trace_bloop(const BatchSlot *__restrict__ slots, WaveBuffers w,
                                                           uint32_t *__restrict__ err, int budget, WaveLoop *L) {
  uint32_t eb = 0;
  const int a = L->iter & 1;
  const int nsh = L->sh[a ^ 1];
  const int next = L->ext[a];
  const int *q = w.queue[a];
  int *fetch = L->fetch + 0;
  const int total = nsh + next;
  const int lane = threadIdx.x & 31;
  int item = -1, pid = 0, pixel = 0, band = 0, dep_band = 0, v = 0;
  bool exhausted = false;
  Traversal t;
  int2 stack[StackSize<W>::value];
  ShadowQuery sq;
  ShadowState ss;
  for (;;) {
    const bool need = item < 0 && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(fetch, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const int idx = base + __popc(m & ((1u << lane) - 1u));
        if (idx >= total) {
          exhausted = true;
        } else if (idx < nsh) {
          item = idx;
          v = w.sq_view[idx];
          const BatchSlot &sl = slots[v];
          const float4 o = w.sq_origin[idx], d = w.sq_dir[idx];
          const int4 mm = w.sq_meta[idx];
          sq.origin = xyz(o);
          sq.max_dist = o.w;
          sq.dir = xyz(d);
          sq.contrib = d.w;
          sq.light_slot = mm.y;
          sq.vol = mm.z;
          pixel = mm.x;
          band = mm.w & 0xff;
          dep_band = mm.w >> 8;
          ss.pos = sq.origin;
          ss.total = 1.f;
          ss.traveled = 0.f;
          ss.vol = sq.vol;
          ss.seg = 0;
          trav_begin(sl.s, t, ss.pos, sq.dir, shadow_bound(sl.s, sl.c, sq, ss, band));
        } else {
          item = idx;
          pid = q[idx - nsh];
          v = w.view[pid];
          const float4 pt = w.pos_thr[pid], ds = w.dir_spdf[pid];
          trav_begin(slots[v].s, t, xyz(pt), xyz(ds), slots[v].c.escape);
        }
      }
    }
    if (__ballot_sync(0xffffffffu, item >= 0) == 0) break;
    const BatchSlot &sl = slots[v];
    if (item >= 0 && trav_advance<W>(sl.s, t, stack, sl.c.eps, budget, eb)) {
      if (item < nsh) {
        if (shadow_segment(sl.s, sl.c, sq, t.h, band, ss)) {
          if (ss.total > 1e-6f) deposit(sl.f, pixel, dep_band, sq.contrib * ss.total, slot_shared(sl));
          item = -1;
        } else {
          trav_begin(sl.s, t, ss.pos, sq.dir, shadow_bound(sl.s, sl.c, sq, ss, band));
        }
      } else {
        w.hit[pid] = make_float4(t.h.t, t.h.u, t.h.v, __int_as_float(t.h.slot));
        item = -1;
      }
    }
  }
  if (eb) atomicOr(err, eb);
}

// shade stage of the batch loop: k_shade_loop with each item's view; an ended
// path's slot starts the next work item of the whole pool, whichever view it
// belongs to
__global__ void __launch_bounds__(kMaxBlock, 4) k_shade_bloop(const BatchSlot *__restrict__ slots, int nslots,
                                                           WaveBuffers w, WaveLoop *L, uint32_t *err) {
  const int a = L->iter & 1;
  const int n = L->ext[a];
  const int *q = w.queue[a];
  int *qn = w.queue[a ^ 1];
  const int total = L->total;
  const bool more = L->next_item < total;
  for (;;) {
    const int base = warp_fetch(L->fetch + 1);
    if (base >= n) break;
    const int i = base + (threadIdx.x & 31);
    Shaded r;
    r.cont = r.nee = false;
    r.pix = -1;
    r.dep_band = 0;
    int pid = -1, v = 0;
    if (i < n) {
      pid = q[i];
      v = w.view[pid];
      const BatchSlot &sl = slots[v];
      const int tag = w.tag[pid];
      const int po = tag >> 16;
      shade_path(sl.s, sl.c, sl.pass0 + (uint32_t)po, slot_band(sl, po), (tag & 0xffff) + 1 >= sl.c.max_depth, sl.f,
                 w, pid, slot_shared(sl), r);
      if (r.cont) w.tag[pid] = tag + 1;
    }
    append_shadow(L->sh + a, w, r, err, v);
    bool fresh = false;
    if (more) {
      const int item = warp_append(&L->next_item, pid >= 0 && !r.cont);
      if (item >= 0 && item < total) {
        start_batch_path(slots, nslots, w, item, pid);
        fresh = true;
      }
    }
    append_ext(L->ext + (a ^ 1), qn, pid, r.cont || fresh, w.capacity, err);
  }
}

}  // namespace

struct BatchLoopGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t capture = nullptr;
};

void free_batch_loop(BatchLoopGraph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->capture) cudaStreamDestroy(g->capture);
  delete g;
}

namespace {

cudaError_t launch_trace_bloop(const BatchSlot *slots, const WaveBuffers &w, uint32_t *err, int width, int grid,
                               int block, int budget, cudaStream_t st) {
  if (width == 9) k_trace_bloop<9><<<grid, block, 0, st>>>(slots, w, err, budget, w.loop);
  else if (width == 5) k_trace_bloop<5><<<grid, block, 0, st>>>(slots, w, err, budget, w.loop);
  else if (width == 8) k_trace_bloop<8><<<grid, block, 0, st>>>(slots, w, err, budget, w.loop);
  else if (width == 4) k_trace_bloop<4><<<grid, block, 0, st>>>(slots, w, err, budget, w.loop);
  else if (width == 3) k_trace_bloop<3><<<grid, block, 0, st>>>(slots, w, err, budget, w.loop);
  else k_trace_bloop<2><<<grid, block, 0, st>>>(slots, w, err, budget, w.loop);
  return cudaGetLastError();
}

// the loop body: one iteration (trace, shade, control)
cudaError_t bloop_body(BatchSlot *slots, int n, const WaveBuffers &w, uint32_t *err, int width, int grid, int block,
                       int budget, cudaGraphConditionalHandle h, int in_graph, cudaStream_t st) {
  cudaError_t e = launch_trace_bloop(slots, w, err, width, grid, block, budget, st);
  if (e != cudaSuccess) return e;
  k_shade_bloop<<<grid, block, 0, st>>>(slots, n, w, w.loop, err);
  k_loop_control<<<1, 32, 0, st>>>(w.loop, h, in_graph, err);
  return cudaGetLastError();
}

cudaError_t bloop_head(BatchSlot *slots, int n, BatchHeader *h, const int *active, const WaveBuffers &w, int capacity,
                       int limit, cudaStream_t st) {
  cudaError_t e = launch_batch_prepare(slots, n, h, active, st);
  if (e != cudaSuccess) return e;
  const int init_grid = (capacity + 255) / 256 < 4096 ? (capacity + 255) / 256 : 4096;
  k_bloop_init<<<init_grid, 256, 0, st>>>(slots, n, h, w, w.loop, capacity, limit);
  return cudaGetLastError();
}

// the whole step as one graph: head -> while(loop body) -> finish
cudaError_t build_bloop_graph(BatchLoopGraph &G, BatchSlot *slots, int n, BatchHeader *h, const int *active,
                              uint32_t *err, const WaveBuffers &w, int width, int grid, int block, int budget,
                              int capacity, int limit, int acc_blocks) {
  cudaError_t e;
  if (!G.capture && (e = cudaStreamCreateWithFlags(&G.capture, cudaStreamNonBlocking)) != cudaSuccess) return e;
  if ((e = cudaGraphCreate(&G.graph, 0)) != cudaSuccess) return e;
  cudaGraphConditionalHandle cond;
  if ((e = cudaGraphConditionalHandleCreate(&cond, G.graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
  // head: prepare + init
  if ((e = cudaStreamBeginCaptureToGraph(G.capture, G.graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return e;
  cudaError_t le = bloop_head(slots, n, h, active, w, capacity, limit, G.capture);
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  std::vector<cudaGraphNode_t> head;
  if (le == cudaSuccess) le = cudaStreamGetCaptureInfo(G.capture, &cs, nullptr, nullptr, &deps, &ndeps);
  if (le == cudaSuccess) head.assign(deps, deps + ndeps);
  cudaGraph_t g2 = nullptr;
  e = cudaStreamEndCapture(G.capture, &g2);
  if (le != cudaSuccess) return le;
  if (e != cudaSuccess) return e;
  // the while-loop
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t loop;
  if ((e = cudaGraphAddNode(&loop, G.graph, head.data(), head.size(), &cp)) != cudaSuccess) return e;
  if ((e = cudaStreamBeginCaptureToGraph(G.capture, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return e;
  le = bloop_body(slots, n, w, err, width, grid, block, budget, cond, 1, G.capture);
  cudaGraph_t body = nullptr;
  e = cudaStreamEndCapture(G.capture, &body);
  if (le != cudaSuccess) return le;
  if (e != cudaSuccess) return e;
  // tail: block averages and pass counters
  if ((e = cudaStreamBeginCaptureToGraph(G.capture, G.graph, &loop, nullptr, 1, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return e;
  le = launch_batch_finish(slots, n, acc_blocks, G.capture);
  e = cudaStreamEndCapture(G.capture, &g2);
  if (le != cudaSuccess) return le;
  if (e != cudaSuccess) return e;
  return cudaGraphInstantiate(&G.exec, G.graph, 0);
}

}  // namespace

cudaError_t launch_batch_loop_step(BatchSlot *slots, int n, BatchHeader *h, const int *active, uint32_t *err,
                                   const WaveBuffers &w, int width, int grid, int block, int budget, int capacity,
                                   int limit, int acc_blocks, cudaStream_t st, BatchLoopGraph **graph,
                                   bool use_graph) {
  if (capacity < 1 || capacity > w.capacity || !w.view || !w.sq_view || !w.tag || !w.loop || limit < 1)
    return cudaErrorInvalidValue;
  if (!use_graph) {
    // the same kernels launched from the host, the loop's continue flag read after each iteration
    cudaError_t e = bloop_head(slots, n, h, active, w, capacity, limit, st);
    if (e != cudaSuccess) return e;
    for (int it = 0; it < limit; ++it) {
      int go = 0;
      e = cudaMemcpyAsync(&go, &w.loop->go, sizeof(int), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return e;
      if (!go) break;
      e = bloop_body(slots, n, w, err, width, grid, block, budget, 0, 0, st);
      if (e != cudaSuccess) return e;
    }
    return launch_batch_finish(slots, n, acc_blocks, st);
  }
  if (!*graph) *graph = new BatchLoopGraph;
  BatchLoopGraph &G = **graph;
  if (!G.exec) {
    const cudaError_t e =
        build_bloop_graph(G, slots, n, h, active, err, w, width, grid, block, budget, capacity, limit, acc_blocks);
    if (e != cudaSuccess) {
      if (G.graph) cudaGraphDestroy(G.graph);
      G.graph = nullptr;
      return e;
    }
  }
  return cudaGraphLaunch(G.exec, st);
}

// ---------------------------------------------------------------------------
// Allocation-free tile pass.
//
// Some callers cannot call cudaMalloc when they render: a host application
// whose device-memory budget is fixed once it has started, or a render loop
// running inside another framework's callbacks where that framework owns the
// allocator.  The regular wavefront pass allocates its path-state buffers on
// first use; this variant takes the same buffers from one fixed, file-scope
// device array instead, so a call allocates nothing.  The price is a bound on
// the work of one call: at most kNoAllocMaxPaths pixels (a tile of the frame).
//
// Every GPU that loads the library holds the array (about 8.4 MB) until the
// process exits.  The CUDA runtime loads the module that holds it lazily: the
// array is reserved on a device by the first call of this entry point there
// (or by an earlier launch of any wavefront kernel of this file), so a host
// with a fixed memory budget makes that first call during start-up.  All calls
// share it: a call clears the counters it needs and
// overwrites the path state it uses, but two calls whose work overlaps on the
// GPU (different streams, or different host threads on one device) race on
// it and must be serialised by the caller.
namespace {

constexpr int kNoAllocMaxPaths = 65536;
constexpr size_t kNaVec = (size_t)kNoAllocMaxPaths * 16;  // one float4/int4 per path
constexpr size_t kNaIdx = (size_t)kNoAllocMaxPaths * 4;   // one int per path
constexpr size_t kNaCounts = 8192 * sizeof(int);
constexpr size_t kNaHist = 2 * kMaxKeys * sizeof(int);
constexpr size_t kNoAllocScratchBytes = 7 * kNaVec + 4 * kNaIdx + kNaCounts + kNaHist;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// camera rays for the pixels of one tile; path slot s <-> pixel
// (x0 + s % tw, y0 + s / tw) of the full frame (pixel ids key the random streams)
__global__ void k_generate_tile(DevScene s, DevConfig c, uint32_t pass, int band, WaveBuffers w, int x0, int y0,
                                int tw, int th) {
  const int n = tw * th;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int i = x0 + p % tw, j = y0 + p / tw;
    const int pixel = j * c.W + i;
    Rng rng;
    rng.init(c.seed, pass, (uint32_t)pixel, c.scene_id);
    PathState ps;
    camera_ray(s, c, i, j, rng, ps, band);
    w.pos_thr[p] = make_float4(ps.pos.x, ps.pos.y, ps.pos.z, ps.thr);
    w.dir_spdf[p] = make_float4(ps.dir.x, ps.dir.y, ps.dir.z, ps.spdf);
    w.meta[p] = make_int4(pixel, band | (band << 8), 0, (int)rng.n);
    w.queue[0][p] = p;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) w.counts[kCntExt + 0] = n;
}

// Device address of the scratch array, looked up once per device and
// context.  The address belongs to the context that loaded this module: after
// a device reset (cudaDeviceReset, or a re-created primary context) the module
// is loaded again elsewhere, so the cached address is keyed on the current
// context and looked up again when it changes.
std::mutex g_noalloc_mutex;
struct NoallocSlot {
  void *ctx = nullptr;  // CUcontext the address was looked up in
  void *ptr = nullptr;
};
NoallocSlot g_noalloc[64];

using CtxGetCurrentFn = int (*)(void **);  // cuCtxGetCurrent, reached through the runtime

CtxGetCurrentFn ctx_get_current() {
  static const CtxGetCurrentFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<CtxGetCurrentFn>(nullptr);
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

}  // namespace

int noalloc_max_paths() { return kNoAllocMaxPaths; }
size_t noalloc_scratch_bytes() { return kNoAllocScratchBytes; }

cudaError_t noalloc_setup(int device, void **ptr) {
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  void *ctx = nullptr;
  const CtxGetCurrentFn get = ctx_get_current();
  const bool known = get && get(&ctx) == 0 && ctx;  // without a context id: look up on every call
  NoallocSlot &slot = g_noalloc[device];
  if (!known || !slot.ptr || slot.ctx != ctx) {
    // the host-side name of the array is only a stand-in; the kernels need
    // the address the device uses, looked up with the device current
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    slot.ptr = p;
    slot.ctx = known ? ctx : nullptr;
  }
  *ptr = slot.ptr;
  return cudaSuccess;
}

cudaError_t launch_wave_tile_noalloc(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                                     void *scratch, int x0, int y0, int tw, int th, uint32_t *err, int grid,
                                     int block, cudaStream_t st, int trace_budget) {
  if (c.max_depth > kMaxDepth) return cudaErrorInvalidValue;
  unsigned char *b = static_cast<unsigned char *>(scratch);
  WaveBuffers w{};
  w.pos_thr = reinterpret_cast<float4 *>(b + 0 * kNaVec);
  w.dir_spdf = reinterpret_cast<float4 *>(b + 1 * kNaVec);
  w.meta = reinterpret_cast<int4 *>(b + 2 * kNaVec);
  w.hit = reinterpret_cast<float4 *>(b + 3 * kNaVec);
  w.sq_origin = reinterpret_cast<float4 *>(b + 4 * kNaVec);
  w.sq_dir = reinterpret_cast<float4 *>(b + 5 * kNaVec);
  w.sq_meta = reinterpret_cast<int4 *>(b + 6 * kNaVec);
  unsigned char *idx = b + 7 * kNaVec;
  w.queue[0] = reinterpret_cast<int *>(idx + 0 * kNaIdx);
  w.queue[1] = reinterpret_cast<int *>(idx + 1 * kNaIdx);
  w.shadow_queue = reinterpret_cast<int *>(idx + 2 * kNaIdx);
  w.sorted = reinterpret_cast<int *>(idx + 3 * kNaIdx);
  w.counts = reinterpret_cast<int *>(idx + 4 * kNaIdx);
  w.key_hist = reinterpret_cast<int *>(idx + 4 * kNaIdx + kNaCounts);
  w.capacity = kNoAllocMaxPaths;
  // the array keeps the previous call's contents: the counters must start at zero
  cudaError_t e = cudaMemsetAsync(w.counts, 0, kNaCounts, st);
  if (e != cudaSuccess) return e;
  const int n = tw * th;
  k_generate_tile<<<(n + 255) / 256, 256, 0, st>>>(s, c, pass, band, w, x0, y0, tw, th);
  for (int d = 0; d < c.max_depth; ++d) {
    launch_trace(s, c, d, f, w, err, grid, block, st, trace_budget);
    k_shade<<<grid, block, 0, st>>>(s, c, pass, band, d, f, w, 0, err);
  }
  if (c.max_depth > 0) launch_trace(s, c, c.max_depth, f, w, err, grid, block, st, trace_budget);
  return cudaGetLastError();
}

}  // namespace ts
