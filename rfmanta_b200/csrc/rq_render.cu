// Whitted frame on the device, one persistent kernel: per pixel the primary
// ray of PinholeCamera::makeRaysSpecialized<true,false> (scalar branch,
// Model/Cameras/PinholeCamera.cc:356-366) with the SingleSampler pixel
// mapping (Engine/PixelSamplers/SingleSampler.cc:38-41), closest-hit
// traversal, the background on a miss (Background::shade), and on a hit
// Lambertian::shade (Model/Materials/Lambertian.cc:63-246) with its shadow
// loop HardShadows::computeShadows (Engine/Shadows/HardShadows.cc:46-360)
// and PointLight::computeLight (Model/Lights/PointLight.cc:31-79): normal,
// face-forwarding, hit position, per light the shadow ray, its any-hit
// traversal and the cosine-weighted accumulation.
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

// Idle lanes a warp gathers before it fetches new pixels.
constexpr int kWhittedRefill = 8;

// The Whitted frame in one persistent kernel: each lane takes a pixel, traces
// its primary ray, and on a hit traces the shadow ray of every point light in
// turn (HardShadows order), accumulating Lambertian::shade; a lane that
// finishes takes the next pixel once kWhittedRefill lanes of its warp are
// idle (one atomic per refill).  Primary and shadow rays share one traversal
// loop (the any-hit rule chosen per lane), so a warp whose lanes are in
// different phases still steps together.  One kernel instead of a primary
// stage, a compaction and a shade stage: a small frame is bound by the
// latency of its slowest pixels, and the stages' tails added up.
template <int KIND, bool STATS>
__global__ void __launch_bounds__(128)
    whitted_fused_kernel(DevScene S, FrameParams P, FrameBuffers B) {
  extern __shared__ int2 smem_stack[];
  RegStack<0> st;
  st.init(smem_stack + threadIdx.x, blockDim.x);
  const int npix = P.xres * P.yres;
  int* counter = &B.counters[kCntWork];
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  const float shadow_tmax = fsub(1.f, kTEpsilon);  // PointLight: 1 - T_EPSILON
  int pix = -1;     // pixel in flight, -1 = idle
  int light = -1;   // -1: primary ray in flight; else this light's shadow ray
  bool exhausted = false;
  Ray r;
  Hit h;
  int ref = kDone;
  float ffn[3], total[3];
  int mat = 0, nshadow = 0;
  Counts cp, cs;
  for (;;) {
    const bool idle = pix < 0 && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, idle);
    const unsigned busy = __ballot_sync(0xffffffffu, pix >= 0);
    if (m != 0u && (__popc(m) >= kWhittedRefill || busy == 0u)) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (idle) {
        const int qi = base + __popc(m & lt_mask);
        if (qi < npix) {
          pix = qi;
          light = -1;
          primary_ray(P, qi % P.xres, qi / P.xres, r);
          int sp;
          start_ray(S, r, h, ref, sp);
          st.sp = 0;
          if (STATS) cp.boxes += 1;
        } else {
          exhausted = true;
        }
      }
    }
    if (__all_sync(0xffffffffu, exhausted)) break;
    if (pix < 0) continue;
    if (ref != kDone) {
      Counts c;
      step_dyn<KIND, 0, STATS>(S, r, h, ref, st, light >= 0, &c);
      if (STATS) {
        if (light < 0) {
          cp.boxes += c.boxes;
          cp.tris += c.tris;
        } else {
          cs.boxes += c.boxes;
          cs.tris += c.tris;
        }
      }
    }
    if (ref != kDone) continue;
    int next;  // first light at or after `next` that sends a shadow ray
    if (light < 0) {
      B.t[pix] = h.t;
      B.prim[pix] = h.id;
      if (h.id < 0) {
        float bg[3];
        background_color(P.env, P.background, r.d, bg);
#pragma unroll
        for (int c = 0; c < 3; ++c) B.rgb[3 * (size_t)pix + c] = bg[c];
        pix = -1;
        continue;
      }
      float nrm[3];
      tri_normal<KIND>(S, h.pos, nrm);
      const float dn = dot3(nrm, r.d);
#pragma unroll
      for (int c = 0; c < 3; ++c) ffn[c] = (dn <= 0.f) ? nrm[c] : -nrm[c];
      ambient_light(P.env, P.ambient, r.d, ffn, total);
      mat = (int)__ldg(S.face_material + h.id);
      // the shadow rays start at the hit point: r.o becomes it below
#pragma unroll
      for (int c = 0; c < 3; ++c) r.o[c] = fadd(r.o[c], fmul(r.d[c], h.t));
      next = 0;
    } else {
      if (h.id < 0) {
        // unshadowed: RayPacket::normalizeDirections, then the cosine term
        float sd[3] = {r.d[0], r.d[1], r.d[2]};
        const float sum = fadd(fadd(fmul(sd[0], sd[0]), fmul(sd[1], sd[1])),
                               fmul(sd[2], sd[2]));
        const float scale = fdiv(1.f, __fsqrt_rn(sum));
#pragma unroll
        for (int c = 0; c < 3; ++c) sd[c] = fmul(sd[c], scale);
        const float cos_theta = dot3(sd, ffn);
        const float* L = P.lights + 6 * light;
#pragma unroll
        for (int c = 0; c < 3; ++c) total[c] = fadd(total[c], fmul(L[3 + c], cos_theta));
      }
      next = light + 1;
    }
    // r.o holds the hit point; find the next light facing it
    light = -1;
    for (int j = next; j < P.n_lights; ++j) {
      const float* L = P.lights + 6 * j;
      const float sd[3] = {fsub(L[0], r.o[0]), fsub(L[1], r.o[1]), fsub(L[2], r.o[2])};
      if (!(dot3(sd, ffn) > 0.f)) continue;  // masked: counts as shadowed
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        r.d[c] = sd[c];
        r.inv[c] = fdiv(1.f, sd[c]);
      }
      r.minT = shadow_tmax;
      light = j;
      break;
    }
    if (light >= 0) {
      ++nshadow;
      int sp;
      start_ray(S, r, h, ref, sp);
      st.sp = 0;
      if (STATS) cs.boxes += 1;
      continue;
    }
    const float* kd = P.materials + 3 * (size_t)mat;
#pragma unroll
    for (int c = 0; c < 3; ++c) B.rgb[3 * (size_t)pix + c] = fmul(total[c], __ldg(kd + c));
    pix = -1;
  }
  int tot = nshadow;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
  if (lane == 0 && tot) atomicAdd(B.shadow_rays_ptr, (unsigned long long)tot);
  if (STATS) {
    flush_counts(B.stats, cp.boxes, cp.tris);
    flush_counts(B.stats + 2, cs.boxes, cs.tris);
  }
}

cudaError_t launch_whitted(const DevScene& S, const FrameParams& P,
                           const FrameBuffers& B, int grid, cudaStream_t st,
                           const cudaEvent_t* ev, int nev) {
  const int bs = 128;
  const size_t smem = (size_t)S.depth * bs * sizeof(int2);
  cudaError_t e = cudaMemsetAsync(B.counters, 0, kNumCounters * sizeof(int), st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(B.shadow_rays_ptr, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  if (nev > 0) cudaEventRecord(ev[0], st);
  const bool stats = B.stats != nullptr;
  if (S.tri_kind == kWald) {
    if (stats) whitted_fused_kernel<kWald, true><<<grid, bs, smem, st>>>(S, P, B);
    else whitted_fused_kernel<kWald, false><<<grid, bs, smem, st>>>(S, P, B);
  } else {
    if (stats) whitted_fused_kernel<kKS, true><<<grid, bs, smem, st>>>(S, P, B);
    else whitted_fused_kernel<kKS, false><<<grid, bs, smem, st>>>(S, P, B);
  }
  if (nev > 1) cudaEventRecord(ev[1], st);
  return cudaGetLastError();
}

int whitted_blocks_per_sm(int tri_kind, size_t smem) {
  const void* f = tri_kind == kWald ? (const void*)whitted_fused_kernel<kWald, false>
                                    : (const void*)whitted_fused_kernel<kKS, false>;
  if (smem > 48 * 1024) {
    const void* all[4] = {(const void*)whitted_fused_kernel<kWald, false>,
                          (const void*)whitted_fused_kernel<kWald, true>,
                          (const void*)whitted_fused_kernel<kKS, false>,
                          (const void*)whitted_fused_kernel<kKS, true>};
    for (const void* g : all)
      cudaFuncSetAttribute(g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, 128, smem);
  return std::max(1, b);
}

}  // namespace rq
