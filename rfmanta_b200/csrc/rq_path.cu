// Path-tracing wavefront (the KajiyaPathtracer loop,
// Engine/Renderers/KajiyaPathtracer.cc:113-302, per path instead of per
// 64-ray packet):
//
//   generate   camera ray per path (pixel, sample): stratified jitter inside
//              the pixel, PinholeCamera basis (PinholeCamera.cc:356-366)
//   per bounce (both stages persistent, warps refilling idle lanes)
//     extend   closest-hit traversal of the live paths (compacted queue)
//     shade    fused stage per live path (the survivors are then compacted
//              in path order, which keeps neighbouring paths together in
//              the next bounce's warps): background on a miss
//              (KajiyaPathtracer.cc:283-291), Lambertian::sampleBSDF cosine
//              sampling (Lambertian.cc:248-280), importance *= reflectance,
//              one area-light sample (AreaLight::computeLight,
//              Model/Lights/AreaLight.cc:25-54, Parallelogram::getRandomPoints)
//              with the HardShadows cull and an any-hit shadow ray traced in
//              the same thread, direct light weighted by the face-forward
//              geometric normal (KajiyaPathtracer.cc:222-234), Russian
//              roulette (russian_roulette_full, KajiyaPathtracer.cc:389-478:
//              kill when rr > max(reflectance); survivors are not rescaled,
//              as in the reference), and
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

// Persistent form of the extension stage: each lane keeps one path's ray in
// flight; after every while-while step the warp counts its idle lanes with a
// ballot and, once `refill` or more are idle (or none is busy), one lane
// claims that many queue entries with a single atomicAdd on the bounce's
// work counter and the idle lanes start them.  Lanes stay busy while a
// warp's rays finish at different times; results do not depend on the
// schedule.
//
// R = traversal-stack entries kept in registers (0, 1, 2 or 4): the newest
// pending children stay in registers and only older ones go to this
// thread's shared-memory column, which holds depth - R entries.
template <int KIND, bool STATS, int R>
__global__ void __launch_bounds__(256)
    path_extend_persistent_kernel(DevScene S, PathParams P, PathBuffers B, int depth, int n0,
                                  int refill) {
  extern __shared__ int2 smem_stack[];
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  RegStack<R> st;
  st.init(stk, stride);
  const int nq = queue_count(B, depth, n0);
  const int* qin = B.queue[depth & 1];
  int* counter = &B.counters[kFetchBase + depth];
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  int p = -1;  // path slot in flight, -1 = idle
  bool exhausted = false;
  Counts cnt;
  Ray r;
  Hit h;
  int ref = kDone;
  for (;;) {
    const bool idle = (p < 0) && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, idle);
    const unsigned busy = __ballot_sync(0xffffffffu, p >= 0);
    if (m != 0u && (__popc(m) >= refill || busy == 0u)) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (idle) {
        const int qi = base + __popc(m & lt_mask);
        if (qi < nq) {
          p = depth == 0 ? qi : qin[qi];
          load_extension_ray(B, p, r);
          start_ray(S, r, h, ref, st.sp);
          st.nreg = 0;
          if (STATS) cnt.boxes += 1;
        } else {
          exhausted = true;
        }
      }
    }
    if (__all_sync(0xffffffffu, exhausted)) break;
    if (p >= 0) {
      if (ref != kDone) step_dyn<KIND, R, STATS>(S, r, h, ref, st, false, &cnt);
      if (ref == kDone) {
        store_extension(P, B, depth, p, r, h);
        p = -1;
      }
    }
  }
  if (STATS) {
    int a = cnt.boxes, b = cnt.tris;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
      atomicAdd(&B.stats[0], (unsigned long long)a);
      atomicAdd(&B.stats[1], (unsigned long long)b);
    }
  }
}

// Persistent form of the shade stage, with the same warp-ballot refill as
// the extension kernel: a lane takes a live path, runs shade_begin, then
// steps its shadow ray's any-hit traversal; when the ray is done (or none was
// needed) it applies shade_finish and the survivors are compacted into the
// next queue at the warp's common point, one atomic per warp.
template <int KIND, bool STATS, int R>
__global__ void __launch_bounds__(256)
    path_shade_persistent_kernel(DevScene S, PathParams P, PathBuffers B, int depth, int n0,
                                 int refill) {
  extern __shared__ int2 smem_stack[];
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  RegStack<R> st;
  st.init(stk, stride);
  const int nq = queue_count(B, depth, n0);
  const int* qin = B.queue[depth & 1];
  int* qout = B.queue[(depth + 1) & 1];
  int* counter = &B.counters[kShadeFetchBase + depth];
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  int p = -1;  // path slot in flight, -1 = idle
  bool exhausted = false, alive = false, traced = false;
  int nshadow = 0;
  Counts cnt;
  float contrib[3];
  Ray sr;
  Hit sh;
  int ref = kDone;
  for (;;) {
    const bool idle = (p < 0) && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, idle);
    const unsigned busy = __ballot_sync(0xffffffffu, p >= 0);
    if (m != 0u && (__popc(m) >= refill || busy == 0u)) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (idle) {
        const int qi = base + __popc(m & lt_mask);
        if (qi < nq) {
          p = depth == 0 ? qi : qin[qi];
          traced = shade_begin<KIND>(S, P, B, depth, p, B.g0 + p, sr, contrib, alive);
          ref = kDone;
          if (traced) {
            ++nshadow;
            start_ray(S, sr, sh, ref, st.sp);
            st.nreg = 0;
            if (STATS) cnt.boxes += 1;
          }
        } else {
          exhausted = true;
        }
      }
    }
    if (__all_sync(0xffffffffu, exhausted)) break;
    bool fin = false;
    if (p >= 0) {
      if (ref != kDone) step_dyn<KIND, R, STATS>(S, sr, sh, ref, st, true, &cnt);
      if (ref == kDone) {
        if (traced && sh.id < 0) shade_finish(B, p, contrib);
        fin = true;
      }
    }
    if (B.alive) {
      if (fin) B.alive[p] = alive ? 1 : 0;
      if (fin) p = -1;
      continue;
    }
    const bool push = fin && alive;
    const unsigned pm = __ballot_sync(0xffffffffu, push);
    if (pm) {
      const int leader = __ffs(pm) - 1;
      int q = 0;
      if ((int)lane == leader) q = atomicAdd(&B.counters[depth + 1], __popc(pm));
      q = __shfl_sync(0xffffffffu, q, leader);
      if (push) qout[q + __popc(pm & lt_mask)] = p;
    }
    if (fin) p = -1;
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

// Ordered compaction of the survivor flags into the next queue (path order):
// per-tile counts, one-block scan of the tile counts (the total becomes the
// next bounce's live count), then every tile writes its survivors in order.
constexpr int kCompactThreads = 256, kCompactPer = 16;
constexpr int kCompactTile = kCompactThreads * kCompactPer;

__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int s = lane < nw ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  total = warp_sums[(blockDim.x >> 5) - 1];
  const int before = warp == 0 ? 0 : warp_sums[warp - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(kCompactThreads)
    compact_count_kernel(const uint8_t* __restrict__ alive, int n, int* tile_counts) {
  __shared__ int ws[32];
  const int base = blockIdx.x * kCompactTile + threadIdx.x * kCompactPer;
  int c = 0;
  for (int k = 0; k < kCompactPer; ++k) c += (base + k < n && alive[base + k]) ? 1 : 0;
  int total;
  block_exclusive_scan(c, ws, total);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024)
    compact_scan_kernel(int* tile_counts, int ntiles, int* total_out) {
  __shared__ int ws[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < ntiles; b0 += blockDim.x) {
    const int i = b0 + threadIdx.x;
    const int v = i < ntiles ? tile_counts[i] : 0;
    int total;
    const int ex = block_exclusive_scan(v, ws, total);
    if (i < ntiles) tile_counts[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total_out = carry;
}

__global__ void __launch_bounds__(kCompactThreads)
    compact_scatter_kernel(const uint8_t* __restrict__ alive, int n,
                           const int* __restrict__ tile_offsets, int* qout) {
  __shared__ int ws[32];
  const int base = blockIdx.x * kCompactTile + threadIdx.x * kCompactPer;
  int c = 0;
  for (int k = 0; k < kCompactPer; ++k) c += (base + k < n && alive[base + k]) ? 1 : 0;
  int total;
  int o = tile_offsets[blockIdx.x] + block_exclusive_scan(c, ws, total);
  for (int k = 0; k < kCompactPer; ++k)
    if (base + k < n && alive[base + k]) qout[o++] = base + k;
}

int flag_compaction_tiles(int n) { return std::max(1, (n + kCompactTile - 1) / kCompactTile); }

cudaError_t launch_flag_compaction(const uint8_t* flags, int n, int* tile_counts, int* total_out,
                                   int* qout, cudaStream_t st) {
  const int tiles = flag_compaction_tiles(n);
  compact_count_kernel<<<tiles, kCompactThreads, 0, st>>>(flags, n, tile_counts);
  compact_scan_kernel<<<1, 1024, 0, st>>>(tile_counts, tiles, total_out);
  compact_scatter_kernel<<<tiles, kCompactThreads, 0, st>>>(flags, n, tile_counts, qout);
  return cudaGetLastError();
}

cudaError_t launch_ordered_compaction(const PathBuffers& B, int n, int depth, cudaStream_t st) {
  const int tiles = std::max(1, (n + kCompactTile - 1) / kCompactTile);
  compact_count_kernel<<<tiles, kCompactThreads, 0, st>>>(B.alive, n, B.tile_counts);
  compact_scan_kernel<<<1, 1024, 0, st>>>(B.tile_counts, tiles, &B.counters[depth + 1]);
  compact_scatter_kernel<<<tiles, kCompactThreads, 0, st>>>(B.alive, n, B.tile_counts,
                                                            B.queue[(depth + 1) & 1]);
  return cudaGetLastError();
}

// Grid of a persistent stage: every SM filled once at the kernel's own
// occupancy for this block size and stack (or blocks_per_sm if smaller).
// With blocks_per_sm below the occupancy maximum, the shared memory the
// resident blocks do not need is left to L1 (the carveout preference is set
// to what those blocks use), so the node and triangle records get more L1.
static int stage_grid(const void* f, int block, int blocks_per_sm, size_t smem) {
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                       cudaSharedmemCarveoutDefault);
  int b = 0, dev = 0, sms = 0, per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, block, smem);
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (blocks_per_sm > 0 && blocks_per_sm < b && per_sm > 0) {
    b = blocks_per_sm;
    const size_t need = (size_t)b * (smem + 1024);  // + the per-block reservation
    const int pct = (int)std::min<size_t>(100, (need * 100 + per_sm - 1) / per_sm);
    cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  }
  return std::max(1, b * sms);
}

// Shared-memory stack bytes per block: the column holds the entries that do
// not fit in the R registers (at least one, so the column is never empty).
static size_t stack_smem(int depth, int block, int regs) {
  return (size_t)std::max(1, depth - regs) * block * sizeof(int2);
}

template <int KIND, bool STATS>
static const void* extend_fn(int regs) {
  return regs == 4 ? (const void*)path_extend_persistent_kernel<KIND, STATS, 4>
       : regs == 2 ? (const void*)path_extend_persistent_kernel<KIND, STATS, 2>
       : regs == 1 ? (const void*)path_extend_persistent_kernel<KIND, STATS, 1>
                   : (const void*)path_extend_persistent_kernel<KIND, STATS, 0>;
}

template <int KIND, bool STATS>
static const void* shade_fn(int regs) {
  return regs == 4 ? (const void*)path_shade_persistent_kernel<KIND, STATS, 4>
       : regs == 2 ? (const void*)path_shade_persistent_kernel<KIND, STATS, 2>
       : regs == 1 ? (const void*)path_shade_persistent_kernel<KIND, STATS, 1>
                   : (const void*)path_shade_persistent_kernel<KIND, STATS, 0>;
}

template <int KIND, bool STATS>
static void launch_bounces(const DevScene& S, const PathParams& P, const PathBuffers& B,
                           int n, const PathLaunch& L, cudaStream_t st,
                           const cudaEvent_t* ev, int nev) {
  const int eb = L.block_threads[0], sb = L.block_threads[1];
  const size_t esm = stack_smem(S.depth, eb, L.reg_stack[0]);
  const size_t ssm = stack_smem(S.depth, sb, L.reg_stack[1]);
  const void* ef = extend_fn<KIND, STATS>(L.reg_stack[0]);
  const void* sf = shade_fn<KIND, STATS>(L.reg_stack[1]);
  const int egrid = stage_grid(ef, eb, L.blocks_per_sm[0], esm);
  const int sgrid = stage_grid(sf, sb, L.blocks_per_sm[1], ssm);
  for (int depth = 0; depth < P.max_depth; ++depth) {
    path_count_kernel<<<1, 32, 0, st>>>(B, depth, n);
    void* eargs[] = {(void*)&S, (void*)&P, (void*)&B, (void*)&depth, (void*)&n,
                     (void*)&L.refill[0]};
    cudaLaunchKernel(ef, dim3(egrid), dim3(eb), eargs, esm, st);
    if (nev > 1 + 2 * depth) cudaEventRecord(ev[1 + 2 * depth], st);
    if (B.alive) cudaMemsetAsync(B.alive, 0, (size_t)n, st);
    void* sargs[] = {(void*)&S, (void*)&P, (void*)&B, (void*)&depth, (void*)&n,
                     (void*)&L.refill[1]};
    cudaLaunchKernel(sf, dim3(sgrid), dim3(sb), sargs, ssm, st);
    if (B.alive) launch_ordered_compaction(B, n, depth, st);
    if (nev > 2 + 2 * depth) cudaEventRecord(ev[2 + 2 * depth], st);
  }
}

cudaError_t launch_path_chunk(const DevScene& S, const PathParams& P, PathBuffers B,
                              long long g0, int n, float* rgb, int grid,
                              const PathLaunch& L, cudaStream_t st, const cudaEvent_t* ev,
                              int nev) {
  B.g0 = g0;
  cudaError_t e = cudaMemsetAsync(B.counters, 0, kPathCounters * sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int ggrid = std::min(grid, (n + 255) / 256);
  path_generate_kernel<<<std::max(ggrid, 1), 256, 0, st>>>(P, B, g0, n);
  if (nev > 0) cudaEventRecord(ev[0], st);
  const bool stats = B.stats != nullptr;
  if (S.tri_kind == kWald) {
    if (stats) launch_bounces<kWald, true>(S, P, B, n, L, st, ev, nev);
    else launch_bounces<kWald, false>(S, P, B, n, L, st, ev, nev);
  } else {
    if (stats) launch_bounces<kKS, true>(S, P, B, n, L, st, ev, nev);
    else launch_bounces<kKS, false>(S, P, B, n, L, st, ev, nev);
  }
  path_resolve_kernel<<<std::max(1, std::min(grid, (n / P.spp + 255) / 256)), 256, 0, st>>>(
      P, B, g0, n, rgb);
  if (nev > 1 + 2 * P.max_depth) cudaEventRecord(ev[1 + 2 * P.max_depth], st);
  return cudaGetLastError();
}

int path_blocks_per_sm(int tri_kind, size_t smem) {
  const void* fs[4] = {(const void*)path_shade_persistent_kernel<kWald, false, 0>,
                       (const void*)path_shade_persistent_kernel<kWald, true, 0>,
                       (const void*)path_shade_persistent_kernel<kKS, false, 0>,
                       (const void*)path_shade_persistent_kernel<kKS, true, 0>};
  if (smem > 48 * 1024)
    for (const void* f : fs)
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fs[tri_kind == kWald ? 0 : 2], 128, smem);
  return std::max(1, b);
}

}  // namespace rq
