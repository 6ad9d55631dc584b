// Triangle record setup: one thread per triangle record, leaf order.
//
// Wald records restate WaldTriangle::setPoints
// (Model/Primitives/WaldTriangle.cc:64-126) with IEEE single-precision
// operations in the same order (no fused multiply-add, correctly rounded
// division and square root), so the stored coefficients equal the
// reference's bit for bit.  Kensler-Shirley records hold p0 and the two
// edges the reference forms per call (KenslerShirleyTriangle.cc:342-347).
#include <cuda_runtime.h>

#include "rq_device.cuh"
#include "rq_internal.h"

namespace rq {

__device__ __forceinline__ float sel3(const float* a, int k) {
  return k == 0 ? a[0] : (k == 1 ? a[1] : a[2]);
}

__global__ void wald_setup_kernel(const float* __restrict__ verts,
                                  const uint32_t* __restrict__ idx,
                                  const int32_t* __restrict__ perm, int n,
                                  float4* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t tag = perm[i];
  const int t = tag & 0x7fffffff;
  float p1[3], p2[3], p3[3];
  const uint32_t i1 = idx[3 * (size_t)t], i2 = idx[3 * (size_t)t + 1],
                 i3 = idx[3 * (size_t)t + 2];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    p1[c] = verts[3 * (size_t)i1 + c];
    p2[c] = verts[3 * (size_t)i2 + c];
    p3[c] = verts[3 * (size_t)i3 + c];
  }
  const float e1[3] = {fsub(p2[0], p1[0]), fsub(p2[1], p1[1]),
                       fsub(p2[2], p1[2])};
  const float e2[3] = {fsub(p3[0], p1[0]), fsub(p3[1], p1[1]),
                       fsub(p3[2], p1[2])};
  float nrm[3];
  cross3(e1, e2, nrm);
  // Vector::normalize (Core/Geometry/Vector.h:322-331)
  const float l = __fsqrt_rn(
      fadd(fadd(fmul(nrm[0], nrm[0]), fmul(nrm[1], nrm[1])),
           fmul(nrm[2], nrm[2])));
  const float scale = fdiv(1.f, l);
  nrm[0] = fmul(nrm[0], scale);
  nrm[1] = fmul(nrm[1], scale);
  nrm[2] = fmul(nrm[2], scale);
  int k = 0;
  if (fabsf(nrm[1]) > fabsf(nrm[0])) k = 1;
  if (fabsf(nrm[2]) > fabsf(sel3(nrm, k))) k = 2;
  const int u = (k == 0) ? 1 : (k == 1 ? 2 : 0);
  const int v = (k == 0) ? 2 : (k == 1 ? 0 : 1);
  const float nk = sel3(nrm, k);
  const float inv_normalk = fdiv(1.f, nk);
  const float n_u = fmul(sel3(nrm, u), inv_normalk);
  const float n_v = fmul(sel3(nrm, v), inv_normalk);
  const float p1u = sel3(p1, u), p1v = sel3(p1, v), p1k = sel3(p1, k);
  const float p2u = sel3(p2, u), p2v = sel3(p2, v);
  const float p3u = sel3(p3, u), p3v = sel3(p3, v);
  const float n_d = fadd(fadd(fmul(p1u, n_u), fmul(p1v, n_v)), p1k);
  float c_nu = fsub(p2v, p1v);
  float c_nv = fadd(-p2u, p1u);
  float c_d = -fadd(fmul(p1u, c_nu), fmul(p1v, c_nv));
  float s = fdiv(1.f, fadd(fadd(fmul(p3u, c_nu), fmul(p3v, c_nv)), c_d));
  c_nu = fmul(c_nu, s);
  c_nv = fmul(c_nv, s);
  c_d = fmul(c_d, s);
  float b_nu = fsub(p3v, p1v);
  float b_nv = fadd(-p3u, p1u);
  float b_d = -fadd(fmul(p1u, b_nu), fmul(p1v, b_nv));
  s = fdiv(1.f, fadd(fadd(fmul(p2u, b_nu), fmul(p2v, b_nv)), b_d));
  b_nu = fmul(b_nu, s);
  b_nv = fmul(b_nv, s);
  b_d = fmul(b_d, s);
  out[3 * (size_t)i + 0] = make_float4(n_u, n_v, n_d, __int_as_float(k));
  out[3 * (size_t)i + 1] = make_float4(b_nu, b_nv, b_d, nk);
  out[3 * (size_t)i + 2] = make_float4(c_nu, c_nv, c_d, __int_as_float(tag));
}

__global__ void ks_setup_kernel(const float* __restrict__ verts,
                                const uint32_t* __restrict__ idx,
                                const int32_t* __restrict__ perm, int n,
                                float4* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t tag = perm[i];
  const int t = tag & 0x7fffffff;
  float p0[3], p1[3], p2[3];
  const uint32_t i0 = idx[3 * (size_t)t], i1 = idx[3 * (size_t)t + 1],
                 i2 = idx[3 * (size_t)t + 2];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    p0[c] = verts[3 * (size_t)i0 + c];
    p1[c] = verts[3 * (size_t)i1 + c];
    p2[c] = verts[3 * (size_t)i2 + c];
  }
  const float e0[3] = {fsub(p1[0], p0[0]), fsub(p1[1], p0[1]),
                       fsub(p1[2], p0[2])};
  const float e1[3] = {fsub(p0[0], p2[0]), fsub(p0[1], p2[1]),
                       fsub(p0[2], p2[2])};
  out[3 * (size_t)i + 0] = make_float4(p0[0], p0[1], p0[2], e0[0]);
  out[3 * (size_t)i + 1] = make_float4(e0[1], e0[2], e1[0], e1[1]);
  out[3 * (size_t)i + 2] = make_float4(e1[2], 0.f, 0.f, __int_as_float(tag));
}

cudaError_t launch_tri_setup(int tri_kind, const float* d_verts,
                             const uint32_t* d_idx, const int32_t* d_perm,
                             int n, float4* d_tris, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int bs = 256;
  const int grid = (n + bs - 1) / bs;
  if (tri_kind == kWald)
    wald_setup_kernel<<<grid, bs, 0, st>>>(d_verts, d_idx, d_perm, n, d_tris);
  else
    ks_setup_kernel<<<grid, bs, 0, st>>>(d_verts, d_idx, d_perm, n, d_tris);
  return cudaGetLastError();
}

}  // namespace rq
