// Device traversal routines shared by the query kernels and the render
// wavefront: exact triangle tests, the pop rule and the while-while step.
// Visit order follows DynBVH::intersectNode (Model/Groups/DynBVH.cc:274-404):
// the child on the near side of the node's split axis first for closest
// hit (dir[axis] > 0 ? left : right), the RTSAH-cheaper child first for any
// hit (isLeftCheaper).  A child whose box was hit but which is visited later
// is pushed with its entry distance; at pop time it is skipped unless
// entry <= current minT, which is exactly the reference's re-test of that
// box at visit time (the box's exit side was already checked at push).
#pragma once

#include "rq_device.cuh"
#include "rq_internal.h"

namespace rq {

template <int KIND>
__device__ __forceinline__ bool tri_test(Ray& r, const float4* p, Hit& h,
                                         bool& last) {
  const float4 a = __ldg(p);
  const float4 b = __ldg(p + 1);
  const float4 c = __ldg(p + 2);
  last = (__float_as_int(c.w) & kLeafEnd) != 0;
  if (KIND == kWald) return wald_test(r, a, b, c, h);
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
  h.pos = -1;
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

// Per-ray traversal counters (the role of DynBVH's COLLECT_STATS,
// Model/Groups/DynBVH.h:314-374): box tests and triangle tests.
struct Counts {
  int boxes = 0;
  int tris = 0;
};

// One while-while step: descend internal records until a leaf is reached
// (or the ray runs out of work), then test that leaf's triangles and pop.
template <int KIND, bool ANY, bool STATS = false>
__device__ __forceinline__ void step(const DevScene& S, Ray& r, Hit& h,
                                     int& ref, int& sp, int2* stk,
                                     int stride, Counts* cnt = nullptr) {
  const bool fast = inv_finite(r);
  while (ref >= 0 && ref != kDone) {
    if (STATS) cnt->boxes += 2;
    const float4* p = S.nodes + 4 * (size_t)ref;
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
    if (STATS) cnt->tris += 1;
    const bool hit = tri_test<KIND>(r, p, h, last);
    if (hit) h.pos = (int)((p - S.tris) / 3);
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
  const int n = a.stride ? a.stride : a.n;
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

}  // namespace rq

namespace rq {

// Traversal stack whose newest R entries (R = 0, 1, 2 or 4) stay in registers
// and whose older entries spill to this thread's shared-memory column (the
// short register stack of a while-while traversal).  LIFO order is kept:
// registers hold the newest entries (r[0] the oldest of them), the shared
// column the older ones.  A spill only happens when all R registers are in
// use, so with at most `depth` pending entries the column never holds more
// than depth - R of them.  Register slots are addressed by selects so the
// array never leaves registers.
template <int R>
struct RegStack {
  static_assert(R == 0 || R == 1 || R == 2 || R == 4, "0, 1, 2 or 4 register entries");
  int2 r0, r1, r2, r3;
  int nreg;
  int sp;
  int2* col;
  int stride;
  __device__ __forceinline__ void init(int2* c, int s) {
    nreg = 0;
    sp = 0;
    col = c;
    stride = s;
  }
  __device__ __forceinline__ void push(int2 e) {
    if (R == 0) {
      col[sp * stride] = e;
      ++sp;
      return;
    }
    if (nreg == R) {
      col[sp * stride] = r0;
      ++sp;
      if (R == 1) {
        r0 = e;
        return;
      }
      r0 = r1;
      if (R == 2) {
        r1 = e;
      } else {
        r1 = r2;
        r2 = r3;
        r3 = e;
      }
      return;
    }
    if (nreg == 0) r0 = e;
    if (R >= 2 && nreg == 1) r1 = e;
    if (R == 4 && nreg == 2) r2 = e;
    if (R == 4 && nreg == 3) r3 = e;
    ++nreg;
  }
  __device__ __forceinline__ bool pop(int2& e) {
    if (R != 0 && nreg > 0) {
      --nreg;
      e = (R == 1 || nreg == 0) ? r0 : r1;
      if (R == 4 && nreg >= 2) e = nreg == 2 ? r2 : r3;
      return true;
    }
    if (sp > 0) {
      --sp;
      e = col[sp * stride];
      return true;
    }
    return false;
  }
};

// Traversal stack split between shared memory and global memory: the first
// `cap` entries of a thread live in its shared-memory column, deeper ones in
// a global-memory area laid out entry-major over all threads of the launch
// (entry k >= cap of thread g at ovf[(k - cap) * ostride + g]).  A kernel can
// then keep a short shared column, so more blocks fit on an SM, and still
// take trees of any depth.  LIFO order as in RegStack.
struct SplitStack {
  int2* col;  // this thread's shared column (stride blockDim.x)
  int cap;
  int2* ovf;  // this thread's first overflow entry (stride = threads of the grid)
  int sp;
  __device__ __forceinline__ void init(int2* c, int k, int2* o) {
    col = c;
    cap = k;
    ovf = o;
    sp = 0;
  }
  __device__ __forceinline__ void push(int2 e) {
    if (sp < cap) col[sp * blockDim.x] = e;
    else ovf[(size_t)(sp - cap) * (gridDim.x * blockDim.x)] = e;
    ++sp;
  }
  __device__ __forceinline__ bool pop(int2& e) {
    if (sp == 0) return false;
    --sp;
    e = sp < cap ? col[sp * blockDim.x] : ovf[(size_t)(sp - cap) * (gridDim.x * blockDim.x)];
    return true;
  }
};

// The while-while step with the any-hit flag decided per ray at run time
// (a warp of the batched kernel may hold closest-hit and any-hit rays of
// different batches and scenes at once) and a RegStack (or a SplitStack).
template <int KIND, int R, bool STATS = false, class Stack = RegStack<R>>
__device__ __forceinline__ void step_dyn(const DevScene& S, Ray& r, Hit& h, int& ref,
                                         Stack& st, bool any, Counts* cnt = nullptr) {
  const bool fast = inv_finite(r);
  while (ref >= 0 && ref != kDone) {
    if (STATS) cnt->boxes += 2;
    const float4* p = S.nodes + 4 * (size_t)ref;
    const float4 q0 = __ldg(p);
    const float4 q1 = __ldg(p + 1);
    const float4 q2 = __ldg(p + 2);
    const int4 q3 = __ldg(reinterpret_cast<const int4*>(p + 3));
    float tl, tr;
    bool hl, hr;
    box_pair(r, fast, q0, q1, q2, hl, hr, tl, tr);
    if (hl && hr) {
      const bool left_first =
          any ? (((q3.z >> 2) & 1) != 0) : (pick3(r.d, q3.z & 3) > 0.f);
      st.push(make_int2(left_first ? q3.y : q3.x, __float_as_int(left_first ? tr : tl)));
      ref = left_first ? q3.x : q3.y;
    } else if (hl) {
      ref = q3.x;
    } else if (hr) {
      ref = q3.y;
    } else {
      ref = kDone;
      int2 e;
      while (st.pop(e))
        if (__int_as_float(e.y) <= r.minT) {
          ref = e.x;
          break;
        }
    }
  }
  if (ref == kDone) return;
  const float4* p = S.tris + 3 * (size_t)(~ref);
  for (;;) {
    bool last;
    if (STATS) cnt->tris += 1;
    const bool hit = tri_test<KIND>(r, p, h, last);
    if (hit) h.pos = (int)((p - S.tris) / 3);
    if (any && hit) {
      ref = kDone;
      return;
    }
    if (last) break;
    p += 3;
  }
  ref = kDone;
  int2 e;
  while (st.pop(e))
    if (__int_as_float(e.y) <= r.minT) {
      ref = e.x;
      break;
    }
}

}  // namespace rq
