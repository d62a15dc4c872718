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

size_t batch_smem_bytes(int n);
cudaError_t batch_set_smem_limit(int n);
// one step: prepare (item ranges), render (persistent pool), accumulate, advance
cudaError_t launch_batch_step(BatchSlot *slots, int n, BatchHeader *h, const int *active, uint32_t *err, int width,
                              int grid, int block, int acc_blocks, cudaStream_t st, int occupancy);

}  // namespace ts
