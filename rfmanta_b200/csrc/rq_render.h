// Frame-level (wavefront) rendering on the device: parameters and buffers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rfmanta_b200.h"
#include "rq_device.cuh"
#include "rq_env.cuh"

namespace rq {

constexpr int kMaxLights = 16;
constexpr int kMaxReflectDepth = 32;  // reflective Phong recursion limit

enum FrameCounter { kCntWork = 0, kNumCounters = 4 };  // kCntWork: pixels handed out

// Per-frame constants (passed by value as a kernel parameter).
struct FrameParams {
  float cam[12];  // eye, lookat-eye, u, v (PinholeCamera::setup basis)
  int xres, yres;
  int n_lights;
  float lights[6 * kMaxLights];  // position xyz, colour rgb
  float ambient[3];
  float background[3];
  Environment env;         // ambient and background kinds
  const float* materials;  // device, 3 floats per material id
  // optional (rq_render_frame): Phong materials, 4 per material id =
  // specular rgb + exponent bits; exponent < 0 = Lambertian.  NULL = all
  // Lambertian.
  const float* phong;
  // optional (rq_render_frame): reflectivity per material id of the Phong
  // materials (NULL = none), with RenderParameters maxDepth and
  // importanceCutoff
  const float* refl;
  int max_depth;
  float cutoff;
};

// Device buffers of one frame.  rgb/t/prim are outputs; the counters are
// scratch.
struct FrameBuffers {
  float* rgb;       // 3 per pixel
  float* t;         // primary hit distance per pixel
  int32_t* prim;    // primary triangle id per pixel (-1 = miss)
  int32_t* counters;                 // scratch: kNumCounters ints
  unsigned long long* shadow_rays_ptr;  // shadow rays sent this frame
  // optional statistics (NULL = off): box tests and triangle tests of the
  // primary rays, then of the shadow rays
  unsigned long long* stats;
};

// Camera ray of pixel (x, y): PinholeCamera::makeRaysSpecialized<true,false>
// scalar branch (Model/Cameras/PinholeCamera.cc:356-366) with the
// SingleSampler pixel mapping (Engine/PixelSamplers/SingleSampler.cc:38-41).
__device__ __forceinline__ void primary_ray(const FrameParams& P, int x, int y,
                                            Ray& r) {
  const float xscale = fdiv(2.f, (float)P.xres);
  const float yscale = fdiv(2.f, (float)P.yres);
  const float xoffset = fmul(fadd(fdiv((float)(-P.xres), 2.f), 0.5f), xscale);
  const float yoffset = fmul(fadd(fdiv((float)(-P.yres), 2.f), 0.5f), yscale);
  const float px = fadd(fmul((float)x, xscale), xoffset);
  const float py = fadd(fmul((float)y, yscale), yoffset);
  float d[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r.o[c] = P.cam[c];
    d[c] = fadd(fadd(fmul(P.cam[9 + c], px), fmul(P.cam[6 + c], py)), P.cam[3 + c]);
  }
  // Vector::normalize (Core/Geometry/Vector.h:322-331)
  const float l = __fsqrt_rn(fadd(fadd(fmul(d[0], d[0]), fmul(d[1], d[1])),
                                  fmul(d[2], d[2])));
  const float s = fdiv(1.f, l);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r.d[c] = fmul(d[c], s);
    r.inv[c] = fdiv(1.f, r.d[c]);
  }
  r.minT = kMaxT;
}

// The frame's one persistent kernel on `grid` blocks of 128 threads; records
// ev[0] before it and ev[1] after it when given.
cudaError_t launch_whitted(const DevScene& S, const FrameParams& P,
                           const FrameBuffers& B, int grid, cudaStream_t st,
                           const cudaEvent_t* ev, int nev);
int whitted_blocks_per_sm(int tri_kind, size_t smem);

// PinholeCamera::setup (Model/Cameras/PinholeCamera.cc:167-198) on the host.
void camera_basis(const float* eye, const float* lookat, const float* up,
                  float hfov, float vfov, float* out12);

// Checks the C ABI's environment and fills the device form (LinearBackground's
// up normalised as its constructor does); false on a bad kind or a zero up.
bool environment_from(const rq_environment& in, Environment& out);

}  // namespace rq
