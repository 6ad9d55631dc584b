// Per-path work of the path-tracing wavefront, shared by the single-frame
// kernels (rq_path.cu) and the served multi-request kernels (rq_serve.cu):
// camera ray generation, closest-hit extension and the fused shade stage.
// Each function handles one path slot; the caller supplies the frame's (or
// the slot's request's) parameters and scene.
#pragma once

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

// Camera ray and fresh state of path slot p (global path id g).
__device__ __forceinline__ void generate_path(const PathParams& P, const PathBuffers& B,
                                              long long g, int p) {
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

// Extension ray of path slot p (o, d of the current bounce, minT = MAXT).
__device__ __forceinline__ void load_extension_ray(const PathBuffers& B, int p, Ray& r) {
  const size_t C = B.capacity;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r.o[c] = B.o[c * C + p];
    r.d[c] = B.d[c * C + p];
    r.inv[c] = fdiv(1.f, r.d[c]);
  }
  r.minT = kMaxT;
}

// Closest hit of path slot p at this bounce (and the optional dump).
__device__ __forceinline__ void store_extension(const PathParams& P, const PathBuffers& B,
                                                int depth, int p, const Ray& r,
                                                const Hit& h) {
  const size_t C = B.capacity;
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

// Closest hit of one live path's current ray.
template <int KIND, bool STATS>
__device__ __forceinline__ void extend_path(const DevScene& S, const PathParams& P,
                                            const PathBuffers& B, int depth, int p,
                                            int2* stk, int stride, Counts& cnt) {
  Ray r;
  load_extension_ray(B, p, r);
  Hit h;
  int ref, sp;
  start_ray(S, r, h, ref, sp);
  if (STATS) cnt.boxes = 1;
  while (ref != kDone) step<KIND, false, STATS>(S, r, h, ref, sp, stk, stride, &cnt);
  store_extension(P, B, depth, p, r, h);
}

// First half of one live path's bounce: background on a miss, else BSDF
// sample, the light sample and Russian roulette, with the path's next state
// (o, d, importance, RNG) written when it survives.  When the light sample
// needs a shadow ray, returns true with the ray in `sr` and the radiance it
// adds when unoccluded in `contrib`; shade_finish then applies it.  `alive`
// tells whether the path continues.
template <int KIND>
__device__ __forceinline__ bool shade_begin(const DevScene& S, const PathParams& P,
                                            const PathBuffers& B, int depth, int p,
                                            long long g, Ray& sr, float* contrib,
                                            bool& alive) {
  const size_t C = B.capacity;
  const bool last_depth = depth + 1 >= P.max_depth;
  const bool do_rr = depth >= P.rr_depth && depth != P.max_depth - 1;
  alive = false;
  bool traced = false;
  float imp[3], o[3], d[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    imp[c] = B.imp[c * C + p];
    o[c] = B.o[c * C + p];
    d[c] = B.d[c * C + p];
  }
  const int prim = B.prim[p];
  if (prim < 0) {
    float bg[3];
    background_color(P.env, P.background, d, bg);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      B.rad[c * C + p] = fadd(B.rad[c * C + p], fmul(bg[c], imp[c]));
    return false;
  }
  Pcg32 rng;
  rng.state = B.rng[p];
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
  if (last_depth) {
    // do_ambient_on_maxdepth (KajiyaPathtracer.cc:259-279): a path still
    // alive after its last bounce is shaded by its material with ambient
    // light only (Lambertian: ambient * kd) times its importance, which
    // already holds this surface's reflectance.  By then sampleBSDF has
    // written the new direction into the packet and the packet's
    // face-forward normals are recomputed against it (the ones sampleBSDF
    // computed lived in a sub-packet's flags), which an EyeAmbient sees.
    float amb[3];
    if (P.env.ambient_kind == kAmbientEye) {
      float fn[3];
      const float dd = dot3(ng, nd);
#pragma unroll
      for (int c = 0; c < 3; ++c) fn[c] = (dd <= 0.f) ? ng[c] : -ng[c];
      ambient_light(P.env, P.ambient, nd, fn, amb);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) amb[c] = P.ambient[c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
      B.rad[c * C + p] = fadd(B.rad[c * C + p], fmul(fmul(amb[c], refl[c]), imp[c]));
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
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      sr.o[c] = hp[c];
      sr.d[c] = ld[c];
      sr.inv[c] = fdiv(1.f, ld[c]);
    }
    sr.minT = fsub(len, kTEpsilon);
    traced = true;
    // what the light adds when the shadow ray is unoccluded
    const float solid_pdf = fmul(P.light_inv_area, fmul(len, len));
    const float f = fdiv(cosine, solid_pdf);
    // RayPacket::normalizeDirections on the shadow ray
    const float sum = fadd(fadd(fmul(ld[0], ld[0]), fmul(ld[1], ld[1])), fmul(ld[2], ld[2]));
    const float s = fdiv(1.f, __fsqrt_rn(sum));
    float ldn[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) ldn[c] = fmul(ld[c], s);
    const float w = dot3(ffn, ldn);
#pragma unroll
    for (int c = 0; c < 3; ++c) contrib[c] = fmul(fmul(imp[c], fmul(f, P.light_color[c])), w);
  }
  alive = !last_depth;
  if (alive && do_rr) {
    // russian_roulette_full (KajiyaPathtracer.cc:389-478) kills a path when
    // rr > max(reflectance) and then applies its 1/max scale to the killed
    // rays it moved past newEnd, not to the survivors: a surviving path keeps
    // its importance unscaled, and so does it here
    const float rr = pcg32_float(rng);
    const float mx = fmaxf(fmaxf(refl[0], refl[1]), refl[2]);
    if (rr > mx) alive = false;
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
  return traced;
}

// Second half: the unoccluded light sample's radiance.
__device__ __forceinline__ void shade_finish(const PathBuffers& B, int p,
                                             const float* contrib) {
  const size_t C = B.capacity;
#pragma unroll
  for (int c = 0; c < 3; ++c) B.rad[c * C + p] = fadd(B.rad[c * C + p], contrib[c]);
}

// One live path at one bounce in one thread: shade_begin, the any-hit
// shadow ray, shade_finish.  Returns true when the path continues.
template <int KIND, bool STATS>
__device__ __forceinline__ bool shade_path(const DevScene& S, const PathParams& P,
                                           const PathBuffers& B, int depth, int p,
                                           long long g, int2* stk, int stride, Counts& cnt,
                                           int& nshadow) {
  Ray sr;
  float contrib[3];
  bool alive;
  if (shade_begin<KIND>(S, P, B, depth, p, g, sr, contrib, alive)) {
    ++nshadow;
    Hit sh;
    int ref, sp;
    start_ray(S, sr, sh, ref, sp);
    if (STATS) cnt.boxes += 1;
    while (ref != kDone) step<KIND, true, STATS>(S, sr, sh, ref, sp, stk, stride, &cnt);
    if (sh.id < 0) shade_finish(B, p, contrib);
  }
  return alive;
}

}  // namespace rq
