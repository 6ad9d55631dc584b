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

#include "rq_path.h"
#include "rq_sample.cuh"
#include "rq_traverse.cuh"

namespace rq {

__device__ __forceinline__ void path_primary(const PathParams& P, long long g,
                                             Pcg32& rng, float* o, float* d) {
  const int spp = P.spp;
  const long long pix = g / spp;
  const int s = (int)(g - pix * spp);
  const int x = (int)(pix % P.xres), y = (int)(pix / P.xres);
  float jx = 0.5f, jy = 0.5f;
  if (spp > 1) {
    const int n = P.strata;
    const int sx = s % n, sy = s / n;
    jx = fdiv(fadd((float)sx, pcg32_float(rng)), (float)n);
    jy = fdiv(fadd((float)sy, pcg32_float(rng)), (float)n);
  }
  const float xscale = fdiv(2.f, (float)P.xres);
  const float yscale = fdiv(2.f, (float)P.yres);
  const float px = fadd(fmul(fadd((float)x, jx), xscale),
                        fmul(fdiv((float)(-P.xres), 2.f), xscale));
  const float py = fadd(fmul(fadd((float)y, jy), yscale),
                        fmul(fdiv((float)(-P.yres), 2.f), yscale));
  float dd[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    o[c] = P.cam[c];
    dd[c] = fadd(fadd(fmul(P.cam[9 + c], px), fmul(P.cam[6 + c], py)), P.cam[3 + c]);
  }
  const float l = __fsqrt_rn(fadd(fadd(fmul(dd[0], dd[0]), fmul(dd[1], dd[1])),
                                  fmul(dd[2], dd[2])));
  const float sc = fdiv(1.f, l);
#pragma unroll
  for (int c = 0; c < 3; ++c) d[c] = fmul(dd[c], sc);
}

__global__ void path_generate_kernel(PathParams P, PathBuffers B, long long g0, int n) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const long long g = g0 + p;
    Pcg32 rng;
    pcg32_seed(rng, P.seed ^ ((unsigned long long)g * 0x9E3779B97F4A7C15ULL),
               (unsigned long long)g);
    float o[3], d[3];
    path_primary(P, g, rng, o, d);
    const size_t C = B.capacity;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      B.o[c * C + p] = o[c];
      B.d[c * C + p] = d[c];
      B.imp[c * C + p] = 1.f;
      B.rad[c * C + p] = 0.f;
    }
    B.rng[p] = rng.state;
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
  const size_t C = B.capacity;
  for (int base = blockIdx.x * blockDim.x; base < nq; base += gridDim.x * blockDim.x) {
    const int qi = base + threadIdx.x;
    Counts cnt;
    if (qi < nq) {
      const int p = depth == 0 ? qi : qin[qi];
      Ray r;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        r.o[c] = B.o[c * C + p];
        r.d[c] = B.d[c * C + p];
        r.inv[c] = fdiv(1.f, r.d[c]);
      }
      r.minT = kMaxT;
      Hit h;
      int ref, sp;
      start_ray(S, r, h, ref, sp);
      if (STATS) cnt.boxes = 1;
      while (ref != kDone) step<KIND, false, STATS>(S, r, h, ref, sp, stk, stride, &cnt);
      B.t[p] = h.t;
      B.pos[p] = h.pos;
      B.prim[p] = h.id;
      if (B.dbg_prim) {
        const size_t k = (size_t)depth * C + p;
        B.dbg_prim[k] = h.id;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          B.dbg_org[(size_t)c * P.max_depth * C + k] = r.o[c];
          B.dbg_dir[(size_t)c * P.max_depth * C + k] = r.d[c];
        }
      }
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

// Geometric normal of the hit triangle record (unit), as in rq_render.cu.
template <int KIND>
__device__ __forceinline__ void record_normal(const DevScene& S, int pos, float* nrm) {
  const float4* p = S.tris + 3 * (size_t)pos;
  if (KIND == kWald) {
    const float4 q0 = __ldg(p);
    const float4 q1 = __ldg(p + 1);
    const int k = __float_as_int(q0.w);
    const float n_k = q1.w;
    const float nu = fmul(n_k, q0.x);
    const float nv = fmul(n_k, q0.y);
    nrm[0] = k == 0 ? n_k : (k == 1 ? nv : nu);
    nrm[1] = k == 1 ? n_k : (k == 2 ? nv : nu);
    nrm[2] = k == 2 ? n_k : (k == 0 ? nv : nu);
  } else {
    const float4 q0 = __ldg(p);
    const float4 q1 = __ldg(p + 1);
    const float4 q2 = __ldg(p + 2);
    const float e0[3] = {q0.w, q1.x, q1.y};
    const float e1[3] = {q1.z, q1.w, q2.x};
    float c[3];
    cross3(e0, e1, c);
    const float sum = fadd(fadd(fmul(c[0], c[0]), fmul(c[1], c[1])), fmul(c[2], c[2]));
    const float scale = fdiv(1.f, __fsqrt_rn(sum));
#pragma unroll
    for (int j = 0; j < 3; ++j) nrm[j] = -fmul(c[j], scale);
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
  const size_t C = B.capacity;
  const unsigned lane = threadIdx.x & 31u;
  const bool last_depth = depth + 1 >= P.max_depth;
  const bool do_rr = depth >= P.rr_depth && depth != P.max_depth - 1;
  for (int base = blockIdx.x * blockDim.x; base < nq; base += gridDim.x * blockDim.x) {
    const int qi = base + threadIdx.x;
    bool alive = false;
    int p = 0;
    int nshadow = 0;
    Counts cnt;
    if (qi < nq) {
      p = depth == 0 ? qi : qin[qi];
      float imp[3], rad[3], o[3], d[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        imp[c] = B.imp[c * C + p];
        rad[c] = B.rad[c * C + p];
        o[c] = B.o[c * C + p];
        d[c] = B.d[c * C + p];
      }
      const int prim = B.prim[p];
      if (prim < 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) rad[c] = fadd(rad[c], fmul(P.background[c], imp[c]));
      } else {
        Pcg32 rng;
        rng.state = B.rng[p];
        const long long g = B.g0 + p;
        rng.inc = ((unsigned long long)g << 1u) | 1u;
        const float t = B.t[p];
        float hp[3], ng[3], ffn[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) hp[c] = fadd(o[c], fmul(d[c], t));
        record_normal<KIND>(S, B.pos[p], ng);
        const float dn = dot3(ng, d);
#pragma unroll
        for (int c = 0; c < 3; ++c) ffn[c] = (dn <= 0.f) ? ng[c] : -ng[c];
        // Lambertian::sampleBSDF
        const float r1 = pcg32_float(rng);
        const float r2 = pcg32_float(rng);
        const float sintheta = __fsqrt_rn(r1);
        const float costheta = __fsqrt_rn(fsub(1.f, r1));
        float cph, sph;
        sincos_2pi(r2, cph, sph);
        const float cosphi = fmul(cph, sintheta);
        const float sinphi = fmul(sph, sintheta);
        float v1[3];
        {  // Vector::findPerpendicular (Core/Geometry/Vector.h:450-462)
          const float d2 = fmul(ffn[2], ffn[2]);
          const float d1 = fmul(ffn[1], ffn[1]);
          if (fadd(d2, d1) < 1e-4f) {
            v1[0] = -ffn[2];
            v1[1] = 0.f;
            v1[2] = ffn[0];
          } else {
            v1[0] = 0.f;
            v1[1] = ffn[2];
            v1[2] = -ffn[1];
          }
          const float l = __fsqrt_rn(fadd(fadd(fmul(v1[0], v1[0]), fmul(v1[1], v1[1])),
                                          fmul(v1[2], v1[2])));
          const float s = fdiv(1.f, l);
#pragma unroll
          for (int c = 0; c < 3; ++c) v1[c] = fmul(v1[c], s);
        }
        float v2[3];
        cross3(v1, ffn, v2);
        float nd[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          nd[c] = fadd(fadd(fmul(ffn[c], costheta), fmul(v1[c], cosphi)), fmul(v2[c], sinphi));
        const float* kd = P.materials + 3 * (size_t)__ldg(S.face_material + prim);
        float refl[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          refl[c] = __ldg(kd + c);
          imp[c] = fmul(imp[c], refl[c]);
        }
        // one area-light sample
        const float lr1 = pcg32_float(rng);
        const float lr2 = pcg32_float(rng);
        float ld[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          ld[c] = fsub(fadd(fadd(P.light_anchor[c], fmul(lr1, P.light_v1[c])),
                            fmul(lr2, P.light_v2[c])),
                       hp[c]);
        const float len = __fsqrt_rn(fadd(fadd(fmul(ld[0], ld[0]), fmul(ld[1], ld[1])),
                                          fmul(ld[2], ld[2])));
        {
          const float s = fdiv(1.f, len);
#pragma unroll
          for (int c = 0; c < 3; ++c) ld[c] = fmul(ld[c], s);
        }
        const float cosine = -dot3(ld, P.light_normal);
        if (cosine > 0.f && dot3(ld, ffn) > 0.f) {
          Ray sr;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            sr.o[c] = hp[c];
            sr.d[c] = ld[c];
            sr.inv[c] = fdiv(1.f, ld[c]);
          }
          sr.minT = fsub(len, kTEpsilon);
          ++nshadow;
          Hit sh;
          int ref, sp;
          start_ray(S, sr, sh, ref, sp);
          if (STATS) cnt.boxes += 1;
          while (ref != kDone) step<KIND, true, STATS>(S, sr, sh, ref, sp, stk, stride, &cnt);
          if (sh.id < 0) {
            const float solid_pdf = fmul(P.light_inv_area, fmul(len, len));
            const float f = fdiv(cosine, solid_pdf);
            // RayPacket::normalizeDirections on the shadow ray
            const float sum = fadd(fadd(fmul(ld[0], ld[0]), fmul(ld[1], ld[1])),
                                   fmul(ld[2], ld[2]));
            const float s = fdiv(1.f, __fsqrt_rn(sum));
            float ldn[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) ldn[c] = fmul(ld[c], s);
            const float w = dot3(ffn, ldn);
#pragma unroll
            for (int c = 0; c < 3; ++c)
              rad[c] = fadd(rad[c], fmul(fmul(imp[c], fmul(f, P.light_color[c])), w));
          }
        }
        alive = !last_depth;
        if (alive && do_rr) {
          const float rr = pcg32_float(rng);
          const float mx = fmaxf(fmaxf(refl[0], refl[1]), refl[2]);
          if (rr > mx) {
            alive = false;
          } else {
            const float sc = fdiv(1.f, mx);
#pragma unroll
            for (int c = 0; c < 3; ++c) imp[c] = fmul(imp[c], sc);
          }
        }
        if (alive) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            B.o[c * C + p] = hp[c];
            B.d[c * C + p] = nd[c];
            B.imp[c * C + p] = imp[c];
          }
          B.rng[p] = rng.state;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) B.rad[c * C + p] = rad[c];
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
