// Whitted frame as a two-stage wavefront on the device:
//
//   stage 1  primary rays: PinholeCamera::makeRaysSpecialized<true,false>
//            scalar branch (Model/Cameras/PinholeCamera.cc:356-366) with the
//            SingleSampler pixel mapping (Engine/PixelSamplers/SingleSampler.cc:
//            38-41), closest-hit traversal, background colour for misses
//            (ConstantBackground::shade), and stream compaction of the hit
//            pixels into a queue (one atomicAdd per warp).
//   stage 2  fused shading over the compacted queue: Lambertian::shade
//            (Model/Materials/Lambertian.cc:63-246) with its shadow loop
//            HardShadows::computeShadows (Engine/Shadows/HardShadows.cc:46-360)
//            and PointLight::computeLight (Model/Lights/PointLight.cc:31-79):
//            normals, face-forwarding, hit position, per light the shadow
//            ray, the any-hit traversal and the cosine-weighted accumulation,
//            all in one thread per shaded pixel.
// All float work keeps the reference's operation order (see rq_device.cuh),
// so colours match the reference's MANTA_SSE=OFF build bit for bit.
#include <cuda_runtime.h>

#include <algorithm>

#include "rq_render.h"
#include "rq_traverse.cuh"

namespace rq {

// Adds a warp's counters into the frame statistics (one atomic per warp).
__device__ __forceinline__ void flush_counts(unsigned long long* dst, int a, int b) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31u) == 0) {
    atomicAdd(dst, (unsigned long long)a);
    atomicAdd(dst + 1, (unsigned long long)b);
  }
}

template <int KIND, bool STATS>
__global__ void __launch_bounds__(128)
    whitted_primary_kernel(DevScene S, FrameParams P, FrameBuffers B) {
  extern __shared__ int2 smem_stack[];
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  const int npix = P.xres * P.yres;
  const unsigned lane = threadIdx.x & 31u;
  // grid-stride over pixels; the loop bound is uniform per block so every
  // lane of a warp reaches the compaction ballot together
  for (int base = blockIdx.x * blockDim.x; base < npix;
       base += gridDim.x * blockDim.x) {
    const int pix = base + threadIdx.x;
    bool hit = false;
    Counts cnt;
    if (pix < npix) {
      const int x = pix % P.xres, y = pix / P.xres;
      Ray r;
      primary_ray(P, x, y, r);
      Hit h;
      int ref, sp;
      start_ray(S, r, h, ref, sp);
      if (STATS) cnt.boxes = 1;
      while (ref != kDone) step<KIND, false, STATS>(S, r, h, ref, sp, stk, stride, &cnt);
      B.t[pix] = h.t;
      B.prim[pix] = h.id;
      B.pos[pix] = h.pos;
      hit = h.id >= 0;
      if (!hit) {
        float bg[3];
        background_color(P.env, P.background, r.d, bg);
#pragma unroll
        for (int c = 0; c < 3; ++c) B.rgb[3 * (size_t)pix + c] = bg[c];
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (m) {
      const int leader = __ffs(m) - 1;
      int q = 0;
      if ((int)lane == leader) q = atomicAdd(&B.counters[kCntQueue], __popc(m));
      q = __shfl_sync(0xffffffffu, q, leader);
      if (hit) B.queue[q + __popc(m & ((1u << lane) - 1u))] = pix;
    }
    if (STATS) flush_counts(B.stats, cnt.boxes, cnt.tris);
  }
}

// Unit geometric normal of the hit triangle from its record: WaldTriangle::
// computeNormal without vertex normals (WaldTriangle.cc:578-590), or the
// KenslerShirleyTriangle cross product (KenslerShirleyTriangle.cc:396-405)
// normalised as RayPacket::computeNormals does (RayPacket.cc:177-186).
template <int KIND>
__device__ __forceinline__ void tri_normal(const DevScene& S, int pos,
                                           float* nrm) {
  const float4* p = S.tris + 3 * (size_t)pos;
  if (KIND == kWald) {
    const float4 q0 = __ldg(p);
    const float4 q1 = __ldg(p + 1);
    const int k = __float_as_int(q0.w);
    const float n_k = q1.w;
    const float nu = fmul(n_k, q0.x);
    const float nv = fmul(n_k, q0.y);
    // normal[k] = n_k, normal[ku] = nu, normal[kv] = nv
    nrm[0] = k == 0 ? n_k : (k == 1 ? nv : nu);
    nrm[1] = k == 1 ? n_k : (k == 2 ? nv : nu);
    nrm[2] = k == 2 ? n_k : (k == 0 ? nv : nu);
  } else {
    const float4 q0 = __ldg(p);
    const float4 q1 = __ldg(p + 1);
    const float4 q2 = __ldg(p + 2);
    const float e0[3] = {q0.w, q1.x, q1.y};
    const float e1[3] = {q1.z, q1.w, q2.x};  // p0 - p2
    float c[3];
    cross3(e0, e1, c);  // Cross(p1-p0, p2-p0) == -c exactly
    const float sum = fadd(fadd(fmul(c[0], c[0]), fmul(c[1], c[1])), fmul(c[2], c[2]));
    const float scale = fdiv(1.f, __fsqrt_rn(sum));
#pragma unroll
    for (int j = 0; j < 3; ++j) nrm[j] = -fmul(c[j], scale);
  }
}

template <int KIND, bool STATS>
__global__ void __launch_bounds__(128)
    whitted_shade_kernel(DevScene S, FrameParams P, FrameBuffers B) {
  extern __shared__ int2 smem_stack[];
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  const int nq = *(volatile const int*)&B.counters[kCntQueue];
  const unsigned lane = threadIdx.x & 31u;
  const float shadow_tmax = fsub(1.f, kTEpsilon);  // PointLight: 1 - T_EPSILON
  for (int base = blockIdx.x * blockDim.x; base < nq; base += gridDim.x * blockDim.x) {
    const int qi = base + threadIdx.x;
    int nshadow = 0;
    Counts cnt;
    if (qi < nq) {
      const int pix = B.queue[qi];
      const int x = pix % P.xres, y = pix / P.xres;
      Ray r;
      primary_ray(P, x, y, r);
      const float t = B.t[pix];
      const int pos = B.pos[pix];
      const int prim = B.prim[pix];
      float nrm[3];
      tri_normal<KIND>(S, pos, nrm);
      const float dn = dot3(nrm, r.d);
      float ffn[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) ffn[c] = (dn <= 0.f) ? nrm[c] : -nrm[c];
      float hp[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) hp[c] = fadd(r.o[c], fmul(r.d[c], t));
      float total[3];
      ambient_light(P.env, P.ambient, r.d, ffn, total);
      for (int j = 0; j < P.n_lights; ++j) {
        const float* L = P.lights + 6 * j;
        float sd[3] = {fsub(L[0], hp[0]), fsub(L[1], hp[1]), fsub(L[2], hp[2])};
        if (!(dot3(sd, ffn) > 0.f)) continue;  // masked: counts as shadowed
        Ray s;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          s.o[c] = hp[c];
          s.d[c] = sd[c];
          s.inv[c] = fdiv(1.f, sd[c]);
        }
        s.minT = shadow_tmax;
        ++nshadow;
        Hit sh;
        int ref, sp;
        start_ray(S, s, sh, ref, sp);
        if (STATS) cnt.boxes += 1;
        while (ref != kDone) step<KIND, true, STATS>(S, s, sh, ref, sp, stk, stride, &cnt);
        if (sh.id >= 0) continue;
        // RayPacket::normalizeDirections (RayPacket.cc:61-71)
        const float sum = fadd(fadd(fmul(sd[0], sd[0]), fmul(sd[1], sd[1])),
                               fmul(sd[2], sd[2]));
        const float scale = fdiv(1.f, __fsqrt_rn(sum));
#pragma unroll
        for (int c = 0; c < 3; ++c) sd[c] = fmul(sd[c], scale);
        const float cos_theta = dot3(sd, ffn);
#pragma unroll
        for (int c = 0; c < 3; ++c) total[c] = fadd(total[c], fmul(L[3 + c], cos_theta));
      }
      const float* kd = P.materials + 3 * (size_t)__ldg(S.face_material + prim);
#pragma unroll
      for (int c = 0; c < 3; ++c) B.rgb[3 * (size_t)pix + c] = fmul(total[c], __ldg(kd + c));
    }
    // one atomic per warp for the shadow-ray count
    int tot = nshadow;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0 && tot) atomicAdd(B.shadow_rays_ptr, (unsigned long long)tot);
    if (STATS) flush_counts(B.stats + 2, cnt.boxes, cnt.tris);
  }
}

cudaError_t launch_whitted(const DevScene& S, const FrameParams& P,
                           const FrameBuffers& B, int grid1, int grid2,
                           cudaStream_t st, const cudaEvent_t* ev, int nev) {
  const int bs = 128;
  const size_t smem = (size_t)S.depth * bs * sizeof(int2);
  cudaError_t e = cudaMemsetAsync(B.counters, 0, kNumCounters * sizeof(int), st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(B.shadow_rays_ptr, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  if (nev > 0) cudaEventRecord(ev[0], st);
  const bool stats = B.stats != nullptr;
  if (S.tri_kind == kWald) {
    if (stats) whitted_primary_kernel<kWald, true><<<grid1, bs, smem, st>>>(S, P, B);
    else whitted_primary_kernel<kWald, false><<<grid1, bs, smem, st>>>(S, P, B);
  } else {
    if (stats) whitted_primary_kernel<kKS, true><<<grid1, bs, smem, st>>>(S, P, B);
    else whitted_primary_kernel<kKS, false><<<grid1, bs, smem, st>>>(S, P, B);
  }
  if (nev > 1) cudaEventRecord(ev[1], st);
  if (S.tri_kind == kWald) {
    if (stats) whitted_shade_kernel<kWald, true><<<grid2, bs, smem, st>>>(S, P, B);
    else whitted_shade_kernel<kWald, false><<<grid2, bs, smem, st>>>(S, P, B);
  } else {
    if (stats) whitted_shade_kernel<kKS, true><<<grid2, bs, smem, st>>>(S, P, B);
    else whitted_shade_kernel<kKS, false><<<grid2, bs, smem, st>>>(S, P, B);
  }
  if (nev > 2) cudaEventRecord(ev[2], st);
  return cudaGetLastError();
}

int whitted_blocks_per_sm(int tri_kind, size_t smem) {
  int a = 0, b = 0;
  const void* f1 = tri_kind == kWald ? (const void*)whitted_primary_kernel<kWald, false>
                                     : (const void*)whitted_primary_kernel<kKS, false>;
  const void* f2 = tri_kind == kWald ? (const void*)whitted_shade_kernel<kWald, false>
                                     : (const void*)whitted_shade_kernel<kKS, false>;
  if (smem > 48 * 1024) {
    const void* all[8] = {(const void*)whitted_primary_kernel<kWald, false>,
                          (const void*)whitted_primary_kernel<kWald, true>,
                          (const void*)whitted_primary_kernel<kKS, false>,
                          (const void*)whitted_primary_kernel<kKS, true>,
                          (const void*)whitted_shade_kernel<kWald, false>,
                          (const void*)whitted_shade_kernel<kWald, true>,
                          (const void*)whitted_shade_kernel<kKS, false>,
                          (const void*)whitted_shade_kernel<kKS, true>};
    for (const void* f : all)
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, f1, 128, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f2, 128, smem);
  return std::max(1, std::min(a, b));
}

}  // namespace rq
