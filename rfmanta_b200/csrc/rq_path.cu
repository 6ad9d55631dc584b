// Path-tracing wavefront (the KajiyaPathtracer loop,
// Engine/Renderers/KajiyaPathtracer.cc:113-302, per path instead of per
// 64-ray packet):
//
//   generate   camera ray per path (pixel, sample): stratified jitter inside
//              the pixel, PinholeCamera basis (PinholeCamera.cc:356-366)
//   per bounce
//     extend   closest-hit traversal of the live paths (compacted queue)
//     shade    fused stage per live path: background on a miss
//              (KajiyaPathtracer.cc:283-291), Lambertian::sampleBSDF cosine
//              sampling (Lambertian.cc:248-280), importance *= reflectance,
//              one area-light sample (AreaLight::computeLight,
//              Model/Lights/AreaLight.cc:25-54, Parallelogram::getRandomPoints)
//              with the HardShadows cull and an any-hit shadow ray traced in
//              the same thread, direct light weighted by the face-forward
//              geometric normal (KajiyaPathtracer.cc:222-234), Russian
//              roulette (russian_roulette_full, KajiyaPathtracer.cc:389-478:
//              kill when rr > max(reflectance), else scale by 1/max), and
//              compaction of the survivors into the next queue
//   resolve    per pixel, the mean of its samples in sample order
//
// Queue sizes live in device memory, so a whole frame is a fixed sequence of
// launches with no host round trip (it can be captured in a CUDA graph).
// Every path draws from its own PCG32 stream keyed by (seed, path id), so a
// path's result does not depend on which other paths share the launch.
#include <cuda_runtime.h>

#include <algorithm>

#include "rq_pathcore.cuh"

namespace rq {

__global__ void path_generate_kernel(PathParams P, PathBuffers B, long long g0, int n) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    generate_path(P, B, g0 + p, p);
  }
}

__device__ __forceinline__ int queue_count(const PathBuffers& B, int depth, int n0) {
  return depth == 0 ? n0 : *(volatile const int*)&B.counters[depth];
}

template <int KIND, bool STATS>
__global__ void __launch_bounds__(128)
    path_extend_kernel(DevScene S, PathParams P, PathBuffers B, int depth, int n0) {
  extern __shared__ int2 smem_stack[];
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  const int nq = queue_count(B, depth, n0);
  const int* qin = B.queue[depth & 1];
  for (int base = blockIdx.x * blockDim.x; base < nq; base += gridDim.x * blockDim.x) {
    const int qi = base + threadIdx.x;
    Counts cnt;
    if (qi < nq) {
      const int p = depth == 0 ? qi : qin[qi];
      extend_path<KIND, STATS>(S, P, B, depth, p, stk, stride, cnt);
    }
    if (STATS) {
      int a = cnt.boxes, b = cnt.tris;
      for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
      }
      if ((threadIdx.x & 31u) == 0) {
        atomicAdd(&B.stats[0], (unsigned long long)a);
        atomicAdd(&B.stats[1], (unsigned long long)b);
      }
    }
  }
}

template <int KIND, bool STATS>
__global__ void __launch_bounds__(128)
    path_shade_kernel(DevScene S, PathParams P, PathBuffers B, int depth, int n0) {
  extern __shared__ int2 smem_stack[];
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  const int nq = queue_count(B, depth, n0);
  const int* qin = B.queue[depth & 1];
  int* qout = B.queue[(depth + 1) & 1];
  const unsigned lane = threadIdx.x & 31u;
  for (int base = blockIdx.x * blockDim.x; base < nq; base += gridDim.x * blockDim.x) {
    const int qi = base + threadIdx.x;
    bool alive = false;
    int p = 0;
    int nshadow = 0;
    Counts cnt;
    if (qi < nq) {
      p = depth == 0 ? qi : qin[qi];
      alive = shade_path<KIND, STATS>(S, P, B, depth, p, B.g0 + p, stk, stride, cnt, nshadow);
    }
    // compaction of the survivors, one atomic per warp
    const unsigned m = __ballot_sync(0xffffffffu, alive);
    if (m) {
      const int leader = __ffs(m) - 1;
      int q = 0;
      if ((int)lane == leader) q = atomicAdd(&B.counters[depth + 1], __popc(m));
      q = __shfl_sync(0xffffffffu, q, leader);
      if (alive) qout[q + __popc(m & ((1u << lane) - 1u))] = p;
    }
    int tot = nshadow;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0 && tot) atomicAdd(&B.ray_counts[1], (unsigned long long)tot);
    if (STATS) {
      int a = cnt.boxes, b = cnt.tris;
      for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
      }
      if (lane == 0) {
        atomicAdd(&B.stats[2], (unsigned long long)a);
        atomicAdd(&B.stats[3], (unsigned long long)b);
      }
    }
  }
}

// Extension rays of this bounce (for the ray count), read on the device.
__global__ void path_count_kernel(PathBuffers B, int depth, int n0) {
  if (threadIdx.x == 0 && blockIdx.x == 0)
    atomicAdd(&B.ray_counts[0], (unsigned long long)queue_count(B, depth, n0));
}

__global__ void path_resolve_kernel(PathParams P, PathBuffers B, long long g0, int n,
                                    float* rgb) {
  const int spp = P.spp;
  const int npix_chunk = n / spp;
  const long long pix0 = g0 / spp;
  const float inv = fdiv(1.f, (float)spp);
  const size_t C = B.capacity;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < npix_chunk;
       k += gridDim.x * blockDim.x) {
    float acc[3] = {0.f, 0.f, 0.f};
    for (int s = 0; s < spp; ++s) {
      const int p = k * spp + s;
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] = fadd(acc[c], B.rad[c * C + p]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) rgb[3 * (size_t)(pix0 + k) + c] = fmul(acc[c], inv);
  }
}

template <int KIND, bool STATS>
static void launch_bounces(const DevScene& S, const PathParams& P, const PathBuffers& B,
                           int n, int grid, size_t smem, cudaStream_t st,
                           const cudaEvent_t* ev, int nev) {
  const int bs = 128;
  for (int depth = 0; depth < P.max_depth; ++depth) {
    path_count_kernel<<<1, 32, 0, st>>>(B, depth, n);
    path_extend_kernel<KIND, STATS><<<grid, bs, smem, st>>>(S, P, B, depth, n);
    if (nev > 1 + 2 * depth) cudaEventRecord(ev[1 + 2 * depth], st);
    path_shade_kernel<KIND, STATS><<<grid, bs, smem, st>>>(S, P, B, depth, n);
    if (nev > 2 + 2 * depth) cudaEventRecord(ev[2 + 2 * depth], st);
  }
}

cudaError_t launch_path_chunk(const DevScene& S, const PathParams& P, PathBuffers B,
                              long long g0, int n, float* rgb, int grid, cudaStream_t st,
                              const cudaEvent_t* ev, int nev) {
  const int bs = 128;
  const size_t smem = (size_t)S.depth * bs * sizeof(int2);
  B.g0 = g0;
  cudaError_t e = cudaMemsetAsync(B.counters, 0, kPathCounters * sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int ggrid = std::min(grid, (n + 255) / 256);
  path_generate_kernel<<<std::max(ggrid, 1), 256, 0, st>>>(P, B, g0, n);
  if (nev > 0) cudaEventRecord(ev[0], st);
  const bool stats = B.stats != nullptr;
  if (S.tri_kind == kWald) {
    if (stats) launch_bounces<kWald, true>(S, P, B, n, grid, smem, st, ev, nev);
    else launch_bounces<kWald, false>(S, P, B, n, grid, smem, st, ev, nev);
  } else {
    if (stats) launch_bounces<kKS, true>(S, P, B, n, grid, smem, st, ev, nev);
    else launch_bounces<kKS, false>(S, P, B, n, grid, smem, st, ev, nev);
  }
  path_resolve_kernel<<<std::max(1, std::min(grid, (n / P.spp + 255) / 256)), 256, 0, st>>>(
      P, B, g0, n, rgb);
  if (nev > 1 + 2 * P.max_depth) cudaEventRecord(ev[1 + 2 * P.max_depth], st);
  return cudaGetLastError();
}

int path_blocks_per_sm(int tri_kind, size_t smem) {
  const void* fs[8] = {(const void*)path_extend_kernel<kWald, false>,
                       (const void*)path_extend_kernel<kWald, true>,
                       (const void*)path_extend_kernel<kKS, false>,
                       (const void*)path_extend_kernel<kKS, true>,
                       (const void*)path_shade_kernel<kWald, false>,
                       (const void*)path_shade_kernel<kWald, true>,
                       (const void*)path_shade_kernel<kKS, false>,
                       (const void*)path_shade_kernel<kKS, true>};
  if (smem > 48 * 1024)
    for (const void* f : fs)
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int a = 0, b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, fs[tri_kind == kWald ? 0 : 2], 128, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fs[tri_kind == kWald ? 4 : 6], 128, smem);
  return std::max(1, std::min(a, b));
}

}  // namespace rq
