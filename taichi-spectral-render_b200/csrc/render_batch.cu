// Batched renderer: many scenes (each a context with its own BVH, materials,
// camera, resolution, depth and film) in one persistent launch per step.
//
// A step renders one whole spectral block (B passes, one per band) of every
// active scene: the work pool is the concatenation of the scenes' B x W x H
// paths, so small frames no longer leave most of the 148 SMs idle and one
// scene's long paths overlap another's short ones.  Each lane finds the scene
// of its work item by binary search in a block-shared copy of the slot table
// and advances its path with the plain megakernel's vertex step
// (mega_path.cuh), so every scene gets exactly the paths ts_render_pass would
// give it.  Pass counters live in device memory and advance on the device,
// so the four kernels of a step (prepare, render, accumulate, advance) are
// captured once as a CUDA graph and replayed step after step.
#include "batch.cuh"
#include "mega_path.cuh"

namespace ts {

namespace {

// per step: work items of each active slot and the pool size; zero the pool counter
__global__ void k_batch_prepare(BatchSlot *slots, int n, BatchHeader *h, const int *__restrict__ active) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int run = 0;
  for (int i = 0; i < n; ++i) {
    BatchSlot &sl = slots[i];
    sl.active = active[i];
    sl.npass = sl.active ? sl.c.B : 0;
    sl.item0 = run;
    sl.items = sl.npass * sl.c.W * sl.c.H;
    run += sl.items;
  }
  h->total = run;
  h->counter = 0;
}

template <int W, int kMinBlocks = 5>
__global__ void __launch_bounds__(128, kMinBlocks) k_render_batch(const BatchSlot *__restrict__ slots, int n,
                                                      BatchHeader *__restrict__ h, uint32_t *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BatchSlot *sh = reinterpret_cast<BatchSlot *>(smem_raw);
  {
    const int words = n * (int)(sizeof(BatchSlot) / 4);
    const uint32_t *src = reinterpret_cast<const uint32_t *>(slots);
    uint32_t *dst = reinterpret_cast<uint32_t *>(smem_raw);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int total = h->total;
  uint32_t errbits = 0;
  bool exhausted = false;
  MegaCounts cnt;
  MegaLane L;
  L.pix = -1;
  int slot = 0;
  for (;;) {
    const bool need = L.pix < 0 && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(&h->counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const int idx = base + __popc(m & ((1u << lane) - 1u));
        if (idx < total) {
          slot = batch_find_slot(sh, n, idx);
          const BatchSlot &sl = sh[slot];
          const int npix = sl.c.W * sl.c.H;
          const int local = idx - sl.item0;
          const int po = local / npix;
          int band = sl.band0 + po;
          if (band >= sl.c.B) band -= sl.c.B;
          mega_start(sl.s, sl.c, L, sl.pass0 + (uint32_t)po, band, local - po * npix);
        } else {
          exhausted = true;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, L.pix >= 0) == 0) break;
    if (L.pix < 0) continue;
    const BatchSlot &sl = sh[slot];
    mega_vertex<W, false>(sl.s, sl.c, sl.f, L, errbits, cnt, true);
  }
  if (errbits) atomicOr(err, errbits);
}

// average_and_reset_block of every scene that rendered this step (grid.y = slot)
__global__ void k_batch_accumulate(const BatchSlot *__restrict__ slots) {
  const BatchSlot &sl = slots[blockIdx.y];
  if (!sl.npass) return;
  const Film f = sl.f;
  const size_t total = (size_t)f.W * f.H * f.B;
  const int n = sl.nblocks + 1;
  const double inv_n = 1.0 / (double)n;
  const double nm1 = (double)(n - 1);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const double b = f.block[i];
    f.mean[i] = (f.mean[i] * nm1 + b) * inv_n;
    f.m2[i] += b * b;
    f.block[i] = 0.0;
  }
}

__global__ void k_batch_advance(BatchSlot *slots, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !slots[i].npass) return;
  slots[i].pass0 += (uint32_t)slots[i].npass;
  slots[i].nblocks += 1;
}

}  // namespace

size_t batch_smem_bytes(int n) { return (size_t)n * sizeof(BatchSlot); }

namespace {
template <int kMin>
void launch_render_batch(BatchSlot *slots, int n, BatchHeader *h, uint32_t *err, int width, int grid, int block,
                         size_t smem, cudaStream_t st) {
  if (width == 9) k_render_batch<9, kMin><<<grid, block, smem, st>>>(slots, n, h, err);
  else if (width == 5) k_render_batch<5, kMin><<<grid, block, smem, st>>>(slots, n, h, err);
  else if (width == 8) k_render_batch<8, kMin><<<grid, block, smem, st>>>(slots, n, h, err);
  else if (width == 4) k_render_batch<4, kMin><<<grid, block, smem, st>>>(slots, n, h, err);
  else if (width == 3) k_render_batch<3, kMin><<<grid, block, smem, st>>>(slots, n, h, err);
  else k_render_batch<2, kMin><<<grid, block, smem, st>>>(slots, n, h, err);
}
}  // namespace

cudaError_t launch_batch_step(BatchSlot *slots, int n, BatchHeader *h, const int *active, uint32_t *err, int width,
                              int grid, int block, int acc_blocks, cudaStream_t st, int occupancy) {
  k_batch_prepare<<<1, 32, 0, st>>>(slots, n, h, active);
  const size_t smem = batch_smem_bytes(n);
  block = block > 128 ? 128 : block;
  if (occupancy >= 8) launch_render_batch<8>(slots, n, h, err, width, grid, block, smem, st);
  else launch_render_batch<5>(slots, n, h, err, width, grid, block, smem, st);
  k_batch_accumulate<<<dim3(acc_blocks, n), 256, 0, st>>>(slots);
  k_batch_advance<<<(n + 127) / 128, 128, 0, st>>>(slots, n);
  return cudaGetLastError();
}

cudaError_t launch_batch_prepare(BatchSlot *slots, int n, BatchHeader *h, const int *active, cudaStream_t st) {
  k_batch_prepare<<<1, 32, 0, st>>>(slots, n, h, active);
  return cudaGetLastError();
}

cudaError_t launch_batch_finish(BatchSlot *slots, int n, int acc_blocks, cudaStream_t st) {
  k_batch_accumulate<<<dim3(acc_blocks, n), 256, 0, st>>>(slots);
  k_batch_advance<<<(n + 127) / 128, 128, 0, st>>>(slots, n);
  return cudaGetLastError();
}

cudaError_t batch_set_smem_limit(int n) {
  const int bytes = (int)batch_smem_bytes(n);
  cudaError_t e = cudaSuccess;
  for (cudaError_t r :
       {cudaFuncSetAttribute(k_render_batch<2, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<3, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<4, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<8, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<5, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<9, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<5, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<9, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<2, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<3, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<4, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
        cudaFuncSetAttribute(k_render_batch<8, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)})
    if (r != cudaSuccess) e = r;
  return e;
}

}  // namespace ts
