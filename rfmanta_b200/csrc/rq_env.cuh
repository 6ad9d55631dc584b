// Ambient light and background of a frame: the constant forms and the
// direction-dependent ones (EyeAmbient, LinearBackground), evaluated in the
// reference's FP32 operation order.
#pragma once

#include "rq_device.cuh"

namespace rq {

enum AmbientKind { kAmbientConstant = 0, kAmbientEye = 1 };
enum BackgroundKind { kBackgroundConstant = 0, kBackgroundLinear = 1 };

// The parts of a frame's lighting setup beyond the ambient and background
// colours themselves (which sit in the frame's parameters).
struct Environment {
  int ambient_kind;
  int background_kind;
  float down[3];  // LinearBackground cdown (cup = the background colour)
  float up[3];    // LinearBackground up, unit length (normalised on the host)
};

// ConstantAmbient::computeAmbient, or EyeAmbient::computeAmbient
// (Model/AmbientLights/EyeAmbient.cc:29-44): colour x cos_theta with
// cos_theta = -Dot(d, N_ff) x (1 - 0.5) + 0.5, where d is the ray's (unit)
// direction and N_ff its face-forward normal.
__device__ __forceinline__ void ambient_light(const Environment& E, const float* color,
                                              const float* d, const float* ffn,
                                              float* out) {
  if (E.ambient_kind == kAmbientEye) {
    const float cos_theta = fadd(fmul(-dot3(d, ffn), 0.5f), 0.5f);
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = fmul(color[c], cos_theta);
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = color[c];
  }
}

// ConstantBackground::shade, or LinearBackground::shade
// (Model/Backgrounds/LinearBackground.cc:28-40): t = 0.5 x (1 + Dot(d, up)),
// colour = cup x t + cdown x (1 - t), d the ray's (unit) direction.
__device__ __forceinline__ void background_color(const Environment& E, const float* cup,
                                                 const float* d, float* out) {
  if (E.background_kind == kBackgroundLinear) {
    const float t = fmul(0.5f, fadd(1.f, dot3(d, E.up)));
    const float s = fsub(1.f, t);
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = fadd(fmul(cup[c], t), fmul(E.down[c], s));
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = cup[c];
  }
}

}  // namespace rq
