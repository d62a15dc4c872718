// Device slot table of the batched renderer (render_batch.cu).
#pragma once
#include "kernels.cuh"

namespace ts {

constexpr int kBatchMaxScenes = 128;  // slots per batch (block-shared copy: ~45 KB at the maximum)

// One scene of a batch.  Written by the host at creation and reset; the step
// kernels keep item0 / items / npass / pass0 / nblocks up to date on the device.
struct __align__(16) BatchSlot {
  DevScene s;
  DevConfig c;
  Film f;
  int item0, items;  // this step's work items [item0, item0 + items)
  uint32_t pass0;    // first pass of the next step
  int npass;         // passes of this step (B when active, else 0)
  int band0;         // band of pass0 (always 0: a step is a whole block)
  int nblocks;       // blocks completed since the last reset
  int active;        // copied from the host-written active flags at each step
  int pad_;
};
static_assert(sizeof(BatchSlot) % 4 == 0, "slot table is copied to shared memory in 32-bit words");

struct BatchHeader {
  int total;    // work items of the current step
  int counter;  // persistent-pool counter
};

// the slot whose work items hold idx: the largest slot whose first item is
// <= idx (an empty slot shares the next one's start and is skipped)
__device__ __forceinline__ int batch_find_slot(const BatchSlot *sl, int n, int idx) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sl[mid].item0 <= idx) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

size_t batch_smem_bytes(int n);
// the first and last kernels of a step, on their own (the batch loop captures
// them around its while-loop): item ranges of the active slots; block
// averages and pass counters of the slots that rendered
cudaError_t launch_batch_prepare(BatchSlot *slots, int n, BatchHeader *h, const int *active, cudaStream_t st);
cudaError_t launch_batch_finish(BatchSlot *slots, int n, int acc_blocks, cudaStream_t st);

// One step of the batch as one regenerating wavefront loop over the work items
// of every active slot (render_wave.cu): prepare, loop init, the while-loop of
// trace -> shade -> control, block averages, pass advance.  With use_graph
// the whole step is one CUDA graph (built at the first step, replayed after);
// limit bounds the loop's iterations (kErrIterationCap past it).
struct BatchLoopGraph;
cudaError_t launch_batch_loop_step(BatchSlot *slots, int n, BatchHeader *h, const int *active, uint32_t *err,
                                   const WaveBuffers &w, int width, int grid, int block, int budget, int capacity,
                                   int limit, int acc_blocks, cudaStream_t st, BatchLoopGraph **graph, bool use_graph);
void free_batch_loop(BatchLoopGraph *g);
cudaError_t batch_set_smem_limit(int n);
// one step: prepare (item ranges), render (persistent pool), accumulate, advance
cudaError_t launch_batch_step(BatchSlot *slots, int n, BatchHeader *h, const int *active, uint32_t *err, int width,
                              int grid, int block, int acc_blocks, cudaStream_t st, int occupancy);

}  // namespace ts
