// Internal interface of the batched traversal kernel (rq_batch.cu), shared
// by batch plans and the render server's ray-query requests.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rq_device.cuh"

namespace rq {

constexpr int kMaxBatchScenes = 32;

// One batch of rays (or a consecutive range of a larger request's rays):
// SoA origins and directions with `stride` elements between the x/y/z rows
// (0 = n), per-ray tmax, outputs indexed like the rays.
struct BatchDesc {
  int scene;
  int n;
  int any;
  int chunk0;  // first chunk index of this batch
  const float* org;
  const float* dir;
  const float* tmax;
  float* t;
  int32_t* prim;
  float* u;
  float* v;
  int stride;
};

struct BatchArgs {
  const DevScene* scenes;
  int n_scenes;
  const BatchDesc* batches;
  int n_batches;
  int total_chunks;
  int chunk_rays;
  int refill;
  int stack_depth;  // shared-memory entries per thread
  int2* ovf;        // split-stack kernels: overflow area (entry-major over the grid's threads)
  int* counter;
  unsigned long long* stats;  // STATS kernels: box tests, triangle tests
};

// The persistent batched kernel (counter must be zero) with `reg_stack`
// register entries (0, 1, 2, 4) and `smem` bytes of stack per block.
cudaError_t launch_batch(int tri_kind, int reg_stack, const BatchArgs& A, int grid, int block,
                         size_t smem, cudaStream_t st);
int batch_blocks_per_sm(int tri_kind, int reg_stack, int block, size_t smem);

}  // namespace rq
