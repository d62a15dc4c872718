// Plain single-scene renderer: one persistent megakernel per launch.
//
// Each lane owns one path (one pixel of cast_rays, main.py:1502-1590) and
// advances it one path vertex per loop iteration (mega_path.cuh).  Lanes whose
// path has ended fetch the next work item with one warp-aggregated atomic, so
// a warp stays full until the pool is exhausted (path regeneration) instead of
// idling behind its longest path.  A launch covers npass consecutive passes
// (a wavelength bundle): work item idx is pixel idx % npix of pass
// pass0 + idx / npix at band (band0 + idx / npix) mod B.  Bands of one launch
// are distinct; fluorescence can still move deposits into another pass's band,
// so multi-pass launches flush with atomics.
#include "mega_path.cuh"

namespace ts {

namespace {

// kCount: also count the work (for the roofline's algorithmic bytes):
// work[0..7] = paths, path vertices, traversals, node visits, triangle tests,
// surface hits resolved, film deposits, (unused).
// kMinBlocks: resident blocks of 128 threads per SM the compiler must allow
// (5: 96 registers, no spills; 8: 64 registers with local-memory spills --
// more warps to hide the node-fetch latency, faster on large frames).
template <int W, bool kCount, int kMinBlocks = 5>
__global__ void __launch_bounds__(128, kMinBlocks) k_render_mega(DevScene s, DevConfig c, uint32_t pass0, int npass, int band0,
                                                     Film f, int *__restrict__ counter, uint32_t *__restrict__ err,
                                                     unsigned long long *__restrict__ work) {
  const int lane = threadIdx.x & 31;
  MegaCounts cnt;
  const int npix = c.W * c.H;
  const int total = npix * npass;
  uint32_t errbits = 0;
  bool exhausted = false;
  MegaLane L;
  L.pix = -1;
  for (;;) {
    const bool need = L.pix < 0 && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const int idx = base + __popc(m & ((1u << lane) - 1u));
        if (idx < total) {
          const int po = idx / npix;
          int band = band0 + po;
          if (band >= c.B) band -= c.B;
          if (kCount) cnt.paths++;
          mega_start(s, c, L, pass0 + (uint32_t)po, band, idx - po * npix, idx);
        } else {
          exhausted = true;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, L.pix >= 0) == 0) break;
    if (L.pix < 0) continue;
    mega_vertex<W, kCount>(s, c, f, L, errbits, cnt, npass > 1);
  }
  if (errbits) atomicOr(err, errbits);
  if (kCount) {
    atomicAdd(work + 0, (unsigned long long)cnt.paths);
    atomicAdd(work + 1, (unsigned long long)cnt.vert);
    atomicAdd(work + 2, (unsigned long long)cnt.trace);
    atomicAdd(work + 3, (unsigned long long)cnt.tc.nodes);
    atomicAdd(work + 4, (unsigned long long)cnt.tc.tris);
    atomicAdd(work + 5, (unsigned long long)cnt.hit);
    atomicAdd(work + 6, (unsigned long long)cnt.dep);
  }
}

template <int W>
void launch_w(const DevScene &s, const DevConfig &c, uint32_t pass0, int npass, int band0, Film f, int *counter,
              uint32_t *err, int grid, int block, cudaStream_t st, unsigned long long *work, int occupancy) {
  if (work) k_render_mega<W, true><<<grid, block, 0, st>>>(s, c, pass0, npass, band0, f, counter, err, work);
  else if (occupancy >= 8)
    k_render_mega<W, false, 8><<<grid, block, 0, st>>>(s, c, pass0, npass, band0, f, counter, err, nullptr);
  else k_render_mega<W, false><<<grid, block, 0, st>>>(s, c, pass0, npass, band0, f, counter, err, nullptr);
}

}  // namespace

cudaError_t launch_render_mega(const DevScene &s, const DevConfig &c, uint32_t pass, int band, Film f,
                               int *counter, uint32_t *err, int grid, int block, cudaStream_t st,
                               unsigned long long *work, int npass, int occupancy) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  block = block > 128 ? 128 : block;  // the kernel is compiled for blocks of at most 128 threads
  if (s.node_width == 9) launch_w<9>(s, c, pass, npass, band, f, counter, err, grid, block, st, work, occupancy);
  else if (s.node_width == 5) launch_w<5>(s, c, pass, npass, band, f, counter, err, grid, block, st, work, occupancy);
  else if (s.node_width == 8) launch_w<8>(s, c, pass, npass, band, f, counter, err, grid, block, st, work, occupancy);
  else if (s.node_width == 4) launch_w<4>(s, c, pass, npass, band, f, counter, err, grid, block, st, work, occupancy);
  else if (c.speculative) launch_w<3>(s, c, pass, npass, band, f, counter, err, grid, block, st, work, occupancy);
  else launch_w<2>(s, c, pass, npass, band, f, counter, err, grid, block, st, work, occupancy);
  return cudaGetLastError();
}

}  // namespace ts
