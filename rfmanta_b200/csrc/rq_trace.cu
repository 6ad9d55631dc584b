// Ray-query traversal kernels: closest hit and any hit over the paired-child
// node records, Wald or Kensler-Shirley triangles.
//
// Visit order follows DynBVH::intersectNode (Model/Groups/DynBVH.cc:274-404):
// the child on the near side of the node's split axis first for closest
// hit (dir[axis] > 0 ? left : right), the RTSAH-cheaper child first for any
// hit (isLeftCheaper).  A child whose box was hit but which is visited
// later is pushed with its entry distance; at pop time it is skipped unless
// entry <= current minT, which is exactly the reference's re-test of that
// box at visit time (the box's exit side was already checked at push).
//
// Two launch forms:
//   * one thread per ray (grid covers the batch);
//   * persistent: a grid sized to fill the GPU once, each warp fetching new
//     rays with one atomicAdd per refill when `refill` or more of its lanes
//     are idle (warp-ballot work stealing).
// The traversal stack lives in shared memory, one column per thread
// (stack[slot * blockDim + tid]), sized to the tree's depth so it can never
// overflow.
#include <cuda_runtime.h>

#include "rq_traverse.cuh"

namespace rq {

template <int KIND, bool ANY>
__global__ void __launch_bounds__(256) trace_kernel(DevScene S, RayArgs a) {
  extern __shared__ int2 smem_stack[];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  Ray r;
  load_ray(a, i, r);
  Hit h;
  int ref, sp;
  start_ray(S, r, h, ref, sp);
  while (ref != kDone) step<KIND, ANY>(S, r, h, ref, sp, stk, stride);
  store_hit(a, i, h);
}

// Persistent form: each lane keeps one ray in flight; after every
// while-while step the warp counts its idle lanes with a ballot and, once
// `refill` or more are idle (or none is busy), one lane claims that many ray
// indices with a single atomicAdd and the idle lanes take them.
template <int KIND, bool ANY>
__global__ void __launch_bounds__(256)
    trace_persistent_kernel(DevScene S, RayArgs a, int* counter, int refill) {
  extern __shared__ int2 smem_stack[];
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  int idx = -1;  // ray in flight, -1 = idle
  bool exhausted = false;
  Ray r;
  Hit h;
  int ref = kDone, sp = 0;
  for (;;) {
    const bool idle = (idx < 0) && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, idle);
    const unsigned busy = __ballot_sync(0xffffffffu, idx >= 0);
    if (m != 0u && (__popc(m) >= refill || busy == 0u)) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (idle) {
        const int mine = base + __popc(m & lt_mask);
        if (mine < a.n) {
          idx = mine;
          load_ray(a, idx, r);
          start_ray(S, r, h, ref, sp);
        } else {
          exhausted = true;
        }
      }
    }
    if (__all_sync(0xffffffffu, exhausted)) break;
    if (idx >= 0) {
      if (ref != kDone) step<KIND, ANY>(S, r, h, ref, sp, stk, stride);
      if (ref == kDone) {
        store_hit(a, idx, h);
        idx = -1;
      }
    }
  }
}

template <int KIND, bool ANY>
static cudaError_t launch_one(const DevScene& S, const RayArgs& a,
                              const LaunchPlan& plan, cudaStream_t st) {
  const size_t smem = (size_t)S.depth * plan.block_threads * sizeof(int2);
  if (!plan.persistent) {
    const int grid = (a.n + plan.block_threads - 1) / plan.block_threads;
    trace_kernel<KIND, ANY><<<grid, plan.block_threads, smem, st>>>(S, a);
  } else {
    trace_persistent_kernel<KIND, ANY>
        <<<plan.grid, plan.block_threads, smem, st>>>(S, a, plan.counter,
                                                      plan.refill);
  }
  return cudaGetLastError();
}

cudaError_t launch_trace(const DevScene& S, const RayArgs& a, bool anyhit,
                         const LaunchPlan& plan, cudaStream_t st) {
  if (a.n <= 0) return cudaSuccess;
  if (S.tri_kind == kWald)
    return anyhit ? launch_one<kWald, true>(S, a, plan, st)
                  : launch_one<kWald, false>(S, a, plan, st);
  return anyhit ? launch_one<kKS, true>(S, a, plan, st)
                : launch_one<kKS, false>(S, a, plan, st);
}

// Occupancy-derived resident blocks per SM for the persistent form.
int max_blocks_per_sm(int tri_kind, bool anyhit, bool persistent,
                      int block_threads, size_t smem) {
  int nb = 0;
  const void* f = nullptr;
  if (tri_kind == kWald)
    f = persistent ? (anyhit ? (const void*)trace_persistent_kernel<kWald, true>
                             : (const void*)trace_persistent_kernel<kWald, false>)
                   : (anyhit ? (const void*)trace_kernel<kWald, true>
                             : (const void*)trace_kernel<kWald, false>);
  else
    f = persistent ? (anyhit ? (const void*)trace_persistent_kernel<kKS, true>
                             : (const void*)trace_persistent_kernel<kKS, false>)
                   : (anyhit ? (const void*)trace_kernel<kKS, true>
                             : (const void*)trace_kernel<kKS, false>);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, block_threads,
                                                    smem) != cudaSuccess)
    return 1;
  return nb > 0 ? nb : 1;
}

}  // namespace rq
