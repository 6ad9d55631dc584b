// Device-side layout and exact float arithmetic of the ray-query path.
//
// HBM layout (built once per scene, read-only while tracing):
//
//   node records   one 64-byte record per internal DynBVH node, holding the
//                  bounds of BOTH children so one visit costs four 128-bit
//                  loads from a single 64-byte-aligned line:
//                    q0 = (L.lo.x, L.lo.y, L.lo.z, L.hi.x)
//                    q1 = (L.hi.y, L.hi.z, R.lo.x, R.lo.y)
//                    q2 = (R.lo.z, R.hi.x, R.hi.y, R.hi.z)
//                    q3 = (L.ref, R.ref, meta, 0)          (int bits)
//                  ref >= 0: index of the child's own record (internal);
//                  ref <  0: leaf whose triangles start at record ~ref.
//                  meta = axis | isLeftCheaper << 2 of the node itself
//                  (DynBVH.h:37-79).
//   triangle       48 bytes per triangle, stored in leaf order so a leaf is
//   records        a contiguous run:
//                    Wald   (WaldTriangle.h:50-64 precompute)
//                      q0 = (n_u, n_v, n_d, k), q1 = (b_nu, b_nv, b_d, n_k),
//                      q2 = (c_nu, c_nv, c_d, id)
//                    Kensler-Shirley (KenslerShirleyTriangle.cc:342-347)
//                      q0 = (p0.xyz, e0.x), q1 = (e0.yz, e1.xy),
//                      q2 = (e1.z, 0, 0, id)   e0 = p1-p0, e1 = p0-p2
//                  id = original triangle index; bit 31 set on the last
//                  triangle of a leaf.
//
// Arithmetic: every float operation goes through __fadd_rn / __fmul_rn /
// __fsub_rn / IEEE division, so no multiply-add is ever fused and each
// result is rounded exactly as the reference's x86-64 SSE scalar code
// rounds it.  Min/max use the reference's ternary forms, which treat NaN
// differently from fminf/fmaxf.
#pragma once

#include <cstdint>

namespace rq {

constexpr float kTEpsilon = 1.e-4f;  // T_EPSILON ((Real)1.e-4)
constexpr float kMaxT = 1.e19f;      // MAXT ((Real)1.e19)
constexpr int kLeafEnd = int(0x80000000u);
constexpr int kMaxDepth = 512;

enum TriKind : int { kWald = 0, kKS = 1 };

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

struct Ray {
  float o[3];
  float d[3];
  float inv[3];
  float minT;
};

// DynBVH::firstIntersects scalar box test (Model/Groups/DynBVH.cc:666-681):
// returns the entry distance when the slab interval is non-empty.
// FAST = true evaluates the reference's ternary min/max with fminf/fmaxf,
// which is exact whenever no slab distance is NaN; that holds for every ray
// whose inverse direction is finite on all three axes (inv_finite), since
// box bounds and origins are finite.  (With t0 == t1 the two forms may pick
// zeros of different sign, which changes neither tmin >= T_EPSILON nor the
// comparison.)
template <bool FAST>
__device__ __forceinline__ bool box_test_t(const Ray& r, float lx, float ly, float lz,
                                           float hx, float hy, float hz, float& tentry) {
  float tmin = kTEpsilon;
  float tmax = r.minT;
  const float lo[3] = {lx, ly, lz};
  const float hi[3] = {hx, hy, hz};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float t0 = fmul(fsub(lo[c], r.o[c]), r.inv[c]);
    const float t1 = fmul(fsub(hi[c], r.o[c]), r.inv[c]);
    if (FAST) {
      tmin = fmaxf(tmin, fminf(t0, t1));
      tmax = fminf(tmax, fmaxf(t0, t1));
    } else {
      const float nr = (t0 < t1) ? t0 : t1;
      const float fr = (t0 < t1) ? t1 : t0;
      tmin = (tmin < nr) ? nr : tmin;
      tmax = (fr < tmax) ? fr : tmax;
    }
  }
  tentry = tmin;
  return tmin <= tmax;
}

__device__ __forceinline__ bool box_test(const Ray& r, float lx, float ly, float lz,
                                         float hx, float hy, float hz, float& tentry) {
  return box_test_t<false>(r, lx, ly, lz, hx, hy, hz, tentry);
}

// Whether box_test_t<true> is exact for this ray (see above).  minT may be
// +inf, which fminf/fmaxf and the ternaries treat alike.
__device__ __forceinline__ bool inv_finite(const Ray& r) {
  return fabsf(r.inv[0]) < INFINITY && fabsf(r.inv[1]) < INFINITY &&
         fabsf(r.inv[2]) < INFINITY && !(r.minT != r.minT);
}

// Both child boxes of a node record (q0..q2) for one ray.
__device__ __forceinline__ void box_pair(const Ray& r, bool fast, const float4& q0,
                                         const float4& q1, const float4& q2, bool& hl,
                                         bool& hr, float& tl, float& tr) {
  if (fast) {
    hl = box_test_t<true>(r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, tl);
    hr = box_test_t<true>(r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, tr);
  } else {
    hl = box_test_t<false>(r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, tl);
    hr = box_test_t<false>(r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, tr);
  }
}

struct Hit {
  float t;
  int id;   // original triangle index, -1 = none
  int pos;  // triangle record index (leaf order) of the hit
  float u, v;
};

__device__ __forceinline__ float pick3(const float* a, int k) {
  return k == 0 ? a[0] : (k == 1 ? a[1] : a[2]);
}

// WaldTriangle::intersect scalar branch (WaldTriangle.cc:489-555) for one
// ray, followed by RayPacket::hit (Interface/RayPacket.h:531-543).  The
// projection axes are chosen with selects so the ray stays in registers.
__device__ __forceinline__ bool wald_test(Ray& r, const float4 q0,
                                          const float4 q1, const float4 q2,
                                          Hit& h) {
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

__device__ __forceinline__ void cross3(const float* a, const float* b,
                                       float* o) {
  o[0] = fsub(fmul(a[1], b[2]), fmul(a[2], b[1]));
  o[1] = fsub(fmul(a[2], b[0]), fmul(a[0], b[2]));
  o[2] = fsub(fmul(a[0], b[1]), fmul(a[1], b[0]));
}

__device__ __forceinline__ float dot3(const float* a, const float* b) {
  return fadd(fadd(fmul(a[0], b[0]), fmul(a[1], b[1])), fmul(a[2], b[2]));
}

// KenslerShirleyTriangle::intersect scalar branch
// (KenslerShirleyTriangle.cc:336-378) for one ray.
__device__ __forceinline__ bool ks_test(Ray& r, const float4 q0,
                                        const float4 q1, const float4 q2,
                                        Hit& h) {
  const float p0[3] = {q0.x, q0.y, q0.z};
  const float e0[3] = {q0.w, q1.x, q1.y};
  const float e1[3] = {q1.z, q1.w, q2.x};
  float n[3];
  cross3(e0, e1, n);
  const float oldt = r.minT;
  const float rcp = fdiv(1.0f, dot3(n, r.d));
  const float e2[3] = {fsub(p0[0], r.o[0]), fsub(p0[1], r.o[1]),
                       fsub(p0[2], r.o[2])};
  const float toverd = fmul(dot3(n, e2), rcp);
  if (toverd > fsub(oldt, kTEpsilon) || toverd < kTEpsilon) return false;
  float im[3];
  cross3(e2, r.d, im);
  const float uoverd = fmul(dot3(im, e1), rcp);
  if (uoverd < 0.0f) return false;
  const float voverd = fmul(dot3(im, e0), rcp);
  if (fadd(uoverd, voverd) > 1.0f || voverd < 0.0f) return false;
  if (toverd > kTEpsilon && toverd < r.minT) {
    r.minT = toverd;
    h.t = toverd;
    h.id = __float_as_int(q2.w) & 0x7fffffff;
    h.u = uoverd;
    h.v = voverd;
    return true;
  }
  return false;
}

// Scene as the kernels see it.
struct DevScene {
  const float4* nodes;  // 4 float4 per record
  const float4* tris;   // 3 float4 per triangle, leaf order
  const uint32_t* face_material;
  int tri_kind;
  int root_ref;  // >= 0 internal record, < 0 leaf (~first)
  float root_lo[3], root_hi[3];
  int depth;  // maximum number of pending stack entries
};

}  // namespace rq
