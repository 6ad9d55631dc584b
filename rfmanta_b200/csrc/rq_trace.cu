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

#include "rq_device.cuh"
#include "rq_internal.h"

namespace rq {

__device__ __forceinline__ float pick3(const float* a, int k) {
  return k == 0 ? a[0] : (k == 1 ? a[1] : a[2]);
}

// Wald test with the axis selection done by selects (no local memory).
__device__ __forceinline__ bool wald_test_sel(Ray& r, const float4 q0,
                                              const float4 q1,
                                              const float4 q2, Hit& h) {
  const int k = __float_as_int(q0.w);
  const int ku = (k == 2) ? 0 : k + 1;
  const int kv = (k == 0) ? 2 : k - 1;
  const float n_u = q0.x, n_v = q0.y, n_d = q0.z;
  const float dk = pick3(r.d, k), dku = pick3(r.d, ku), dkv = pick3(r.d, kv);
  const float ok = pick3(r.o, k), oku = pick3(r.o, ku), okv = pick3(r.o, kv);
  const float nd0 = fadd(fadd(fmul(n_u, dku), fmul(n_v, dkv)), dk);
  const float nd = fdiv(1.f, nd0);
  const float f0 = fsub(n_d, fadd(fadd(ok, fmul(n_u, oku)), fmul(n_v, okv)));
  const float f = fmul(f0, nd);
  if (f < kTEpsilon || f > r.minT) return false;
  const float hu = fadd(oku, fmul(f, dku));
  const float hv = fadd(okv, fmul(f, dkv));
  const float lambda = fadd(fadd(q1.z, fmul(hu, q1.x)), fmul(hv, q1.y));
  if (lambda < 0.f) return false;
  const float mue = fadd(fadd(q2.z, fmul(hu, q2.x)), fmul(hv, q2.y));
  if (mue < 0.f || fadd(mue, lambda) > 1.f) return false;
  if (f > kTEpsilon && f < r.minT) {
    r.minT = f;
    h.t = f;
    h.id = __float_as_int(q2.w) & 0x7fffffff;
    h.u = lambda;
    h.v = mue;
    return true;
  }
  return false;
}

template <int KIND>
__device__ __forceinline__ bool tri_test(Ray& r, const float4* p, Hit& h,
                                         bool& last) {
  const float4 a = __ldg(p);
  const float4 b = __ldg(p + 1);
  const float4 c = __ldg(p + 2);
  last = (__float_as_int(c.w) & kLeafEnd) != 0;
  if (KIND == kWald) return wald_test_sel(r, a, b, c, h);
  return ks_test(r, a, b, c, h);
}

constexpr int kDone = 0x7fffffff;

// Pops the next pending child whose entry distance still lies within minT;
// ref = kDone when nothing is left.
__device__ __forceinline__ void pop(const Ray& r, int& ref, int& sp,
                                    const int2* stk, int stride) {
  for (;;) {
    if (sp == 0) {
      ref = kDone;
      return;
    }
    --sp;
    const int2 e = stk[sp * stride];
    if (__int_as_float(e.y) <= r.minT) {
      ref = e.x;
      return;
    }
  }
}

// Root box test (firstIntersects on nodes[0].bounds); sets ref.
__device__ __forceinline__ void start_ray(const DevScene& S, const Ray& r,
                                          Hit& h, int& ref, int& sp) {
  h.id = -1;
  h.t = r.minT;
  h.u = 0.f;
  h.v = 0.f;
  sp = 0;
  float te;
  ref = box_test(r, S.root_lo[0], S.root_lo[1], S.root_lo[2], S.root_hi[0],
                 S.root_hi[1], S.root_hi[2], te)
            ? S.root_ref
            : kDone;
}

// One while-while step: descend internal records until a leaf is reached
// (or the ray runs out of work), then test that leaf's triangles and pop.
template <int KIND, bool ANY>
__device__ __forceinline__ void step(const DevScene& S, Ray& r, Hit& h,
                                     int& ref, int& sp, int2* stk,
                                     int stride) {
  while (ref >= 0 && ref != kDone) {
    const float4* p = S.nodes + 4 * (size_t)ref;
    const float4 q0 = __ldg(p);
    const float4 q1 = __ldg(p + 1);
    const float4 q2 = __ldg(p + 2);
    const int4 q3 = __ldg(reinterpret_cast<const int4*>(p + 3));
    float tl, tr;
    const bool hl = box_test(r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, tl);
    const bool hr = box_test(r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, tr);
    if (hl && hr) {
      const bool left_first =
          ANY ? (((q3.z >> 2) & 1) != 0) : (pick3(r.d, q3.z & 3) > 0.f);
      const int first = left_first ? q3.x : q3.y;
      const int second = left_first ? q3.y : q3.x;
      const float ts = left_first ? tr : tl;
      stk[sp * stride] = make_int2(second, __float_as_int(ts));
      ++sp;
      ref = first;
    } else if (hl) {
      ref = q3.x;
    } else if (hr) {
      ref = q3.y;
    } else {
      pop(r, ref, sp, stk, stride);
    }
  }
  if (ref == kDone) return;
  // leaf
  const float4* p = S.tris + 3 * (size_t)(~ref);
  for (;;) {
    bool last;
    const bool hit = tri_test<KIND>(r, p, h, last);
    if (ANY && hit) {
      ref = kDone;
      return;
    }
    if (last) break;
    p += 3;
  }
  pop(r, ref, sp, stk, stride);
}

__device__ __forceinline__ void load_ray(const RayArgs& a, int i, Ray& r) {
  const int n = a.n;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r.o[c] = __ldg(a.org + (size_t)c * n + i);
    r.d[c] = __ldg(a.dir + (size_t)c * n + i);
    r.inv[c] = fdiv(1.f, r.d[c]);  // RayPacket.cc:106-110
  }
  r.minT = __ldg(a.tmax + i);
}

__device__ __forceinline__ void store_hit(const RayArgs& a, int i,
                                          const Hit& h) {
  if (a.t) a.t[i] = h.t;
  if (a.prim) a.prim[i] = h.id;
  if (a.u) a.u[i] = h.u;
  if (a.v) a.v[i] = h.v;
}

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
