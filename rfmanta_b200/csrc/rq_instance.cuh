// Two-level traversal: a top-level tree over translated instances of
// inner scenes (InstanceT, Model/Instances/InstanceT.cc:60-90).
//
// At a top-level leaf every instance in turn gets the ray with its origin
// moved into the instance (o - translation, the same direction, inverse
// direction and the current minT), the inner scene is traversed in full on
// the same stack above the pending top-level entries, and a hit lowers the
// shared minT, exactly as InstanceT hands its packet to the inner
// DynBVH::intersect and accepts the result through RayPacket::hit.
#pragma once

#include "rq_traverse.cuh"

namespace rq {

// With STATS, cnt counts box tests (two per top-level record, one per root
// box, the instance's included) and triangle tests.
template <int KIND, bool ANY, bool STATS = false>
__device__ __forceinline__ void trace_two_level(const DevScene& T, const DevScene* blas,
                                                Ray& r, Hit& h, int& inst_hit, int& blas_hit,
                                                int2* stk, int stride, Counts* cnt = nullptr) {
  h.id = -1;
  h.pos = -1;
  h.t = r.minT;
  h.u = h.v = 0.f;
  inst_hit = -1;
  blas_hit = -1;
  float te;
  if (STATS) cnt->boxes += 1;
  if (!box_test(r, T.root_lo[0], T.root_lo[1], T.root_lo[2], T.root_hi[0], T.root_hi[1],
                T.root_hi[2], te))
    return;
  int ref = T.root_ref;
  int sp = 0;
  const bool fast = inv_finite(r);
  for (;;) {
    while (ref >= 0 && ref != kDone) {
      if (STATS) cnt->boxes += 2;
      const float4* p = T.nodes + 4 * (size_t)ref;
      const float4 q0 = __ldg(p);
      const float4 q1 = __ldg(p + 1);
      const float4 q2 = __ldg(p + 2);
      const int4 q3 = __ldg(reinterpret_cast<const int4*>(p + 3));
      float tl, tr;
      bool hl, hr;
      box_pair(r, fast, q0, q1, q2, hl, hr, tl, tr);
      if (hl && hr) {
        const bool left_first =
            ANY ? (((q3.z >> 2) & 1) != 0) : (pick3(r.d, q3.z & 3) > 0.f);
        stk[sp * stride] = make_int2(left_first ? q3.y : q3.x,
                                     __float_as_int(left_first ? tr : tl));
        ++sp;
        ref = left_first ? q3.x : q3.y;
      } else if (hl) {
        ref = q3.x;
      } else if (hr) {
        ref = q3.y;
      } else {
        pop(r, ref, sp, stk, stride);
      }
    }
    if (ref == kDone) return;
    const float4* ip = T.tris + 2 * (size_t)(~ref);
    for (;;) {
      const float4 a = __ldg(ip);
      const float4 b = __ldg(ip + 1);
      const int tag = __float_as_int(b.x);
      // an any-hit query ignores InstanceT objects (see rq_scene_create_instanced)
      if (ANY && __float_as_int(b.y) == 0) {
        if (tag & kLeafEnd) break;
        ip += 2;
        continue;
      }
      const DevScene& S = blas[__float_as_int(a.w)];
      Ray lr;
      lr.o[0] = fsub(r.o[0], a.x);
      lr.o[1] = fsub(r.o[1], a.y);
      lr.o[2] = fsub(r.o[2], a.z);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lr.d[c] = r.d[c];
        lr.inv[c] = r.inv[c];
      }
      lr.minT = r.minT;
      Hit lh;
      int lref, lsp;
      if (STATS) cnt->boxes += 1;
      start_ray(S, lr, lh, lref, lsp);
      while (lref != kDone)
        step<KIND, ANY, STATS>(S, lr, lh, lref, lsp, stk + sp * stride, stride, cnt);
      if (lh.id >= 0) {
        r.minT = lr.minT;
        h = lh;
        inst_hit = tag & 0x7fffffff;
        blas_hit = __float_as_int(a.w);
        if (ANY) return;
      }
      if (tag & kLeafEnd) break;
      ip += 2;
    }
    pop(r, ref, sp, stk, stride);
    if (ref == kDone) return;
  }
}

}  // namespace rq
