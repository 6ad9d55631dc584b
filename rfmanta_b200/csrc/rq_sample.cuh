// Sampling helpers of the path-tracing wavefront, written so the CPU
// restatement can repeat them bit for bit:
//   * PCG32 (O'Neill 2014, "PCG: A Family of Simple Fast Space-Efficient
//     Statistically Good Algorithms for Random Number Generation"),
//     pcg32_srandom_r / pcg32_random_r, integer only;
//   * uniform floats in [0, 1) from the top 24 bits;
//   * sin/cos of 2*pi*u for u in [0, 1): quadrant index from 4u (exact),
//     the remainder angle y in [0, pi/2) and Taylor polynomials of sin
//     (degree 11) and cos (degree 12) in Horner form, every operation a
//     separately rounded float add or multiply.  Maximum error below 2e-7
//     over [0, 1) (checked against CUDA's sincosf in the tests).
#pragma once

#include <cstdint>

#include "rq_device.cuh"

namespace rq {

struct Pcg32 {
  uint64_t state;
  uint64_t inc;
};

__device__ __forceinline__ uint32_t pcg32_next(Pcg32& g) {
  const uint64_t old = g.state;
  g.state = old * 6364136223846793005ULL + g.inc;
  const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  const uint32_t rot = (uint32_t)(old >> 59u);
  return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
}

__device__ __forceinline__ void pcg32_seed(Pcg32& g, uint64_t initstate,
                                           uint64_t initseq) {
  g.state = 0u;
  g.inc = (initseq << 1u) | 1u;
  pcg32_next(g);
  g.state += initstate;
  pcg32_next(g);
}

__device__ __forceinline__ float pcg32_float(Pcg32& g) {
  return (float)(pcg32_next(g) >> 8) * (1.0f / 16777216.0f);
}

// (cos, sin) of 2*pi*u, u in [0, 1).
__device__ __forceinline__ void sincos_2pi(float u, float& c, float& s) {
  const float u4 = fmul(u, 4.f);             // exact
  const float qf = floorf(u4);
  const int q = (int)qf & 3;
  const float f = fsub(u4, qf);              // exact
  const float y = fmul(f, 1.57079632679489662f);
  const float y2 = fmul(y, y);
  // sin(y) = y (1 - y2/6 (1 - y2/20 (1 - y2/42 (1 - y2/72 (1 - y2/110)))))
  float ps = fsub(1.f, fmul(y2, 1.f / 110.f));
  ps = fsub(1.f, fmul(fmul(y2, 1.f / 72.f), ps));
  ps = fsub(1.f, fmul(fmul(y2, 1.f / 42.f), ps));
  ps = fsub(1.f, fmul(fmul(y2, 1.f / 20.f), ps));
  ps = fsub(1.f, fmul(fmul(y2, 1.f / 6.f), ps));
  const float sy = fmul(y, ps);
  // cos(y) = 1 - y2/2 (1 - y2/12 (1 - y2/30 (1 - y2/56 (1 - y2/90 (1 - y2/132)))))
  float pc = fsub(1.f, fmul(y2, 1.f / 132.f));
  pc = fsub(1.f, fmul(fmul(y2, 1.f / 90.f), pc));
  pc = fsub(1.f, fmul(fmul(y2, 1.f / 56.f), pc));
  pc = fsub(1.f, fmul(fmul(y2, 1.f / 30.f), pc));
  pc = fsub(1.f, fmul(fmul(y2, 1.f / 12.f), pc));
  const float cy = fsub(1.f, fmul(fmul(y2, 0.5f), pc));
  switch (q) {
    case 0: c = cy; s = sy; break;
    case 1: c = -sy; s = cy; break;
    case 2: c = -cy; s = -sy; break;
    default: c = sy; s = -cy; break;
  }
}

}  // namespace rq
