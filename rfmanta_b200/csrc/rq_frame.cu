// Frame entry points of the C ABI: camera basis and the Whitted wavefront.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/rfmanta_b200.h"
#include "rq_render.h"
#include "rq_scene.h"

namespace rq {

static float hsqrt(float x) { return std::sqrt(x); }

static void hnormalize(float* a) {
  const float l = hsqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  const float s = 1 / l;
  a[0] *= s;
  a[1] *= s;
  a[2] *= s;
}

static void hcross(const float* a, const float* b, float* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// PinholeCamera::setup (Model/Cameras/PinholeCamera.cc:167-198): the
// field-of-view tangents are evaluated in double (DtoR, tan) and stored as
// float, everything else is float.
void camera_basis(const float* eye, const float* lookat, const float* up_in,
                  float hfov, float vfov, float* out) {
  float dir[3] = {lookat[0] - eye[0], lookat[1] - eye[1], lookat[2] - eye[2]};
  const float nearZ = hsqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  float up[3] = {up_in[0], up_in[1], up_in[2]};
  hnormalize(up);
  float v[3], u[3];
  hcross(dir, up, v);
  hnormalize(v);
  hcross(v, dir, u);
  hnormalize(u);
  const double kPi = 3.14159265358979323846;
  const float height = (float)(nearZ * std::tan((0.5 * vfov) * (kPi / 180.)));
  for (int c = 0; c < 3; ++c) u[c] *= height;
  const float width = (float)(nearZ * std::tan((0.5 * hfov) * (kPi / 180.)));
  for (int c = 0; c < 3; ++c) v[c] *= width;
  for (int c = 0; c < 3; ++c) {
    out[c] = eye[c];
    out[3 + c] = dir[c];
    out[6 + c] = u[c];
    out[9 + c] = v[c];
  }
}

bool environment_from(const rq_environment& in, Environment& out) {
  std::memset(&out, 0, sizeof(out));
  if (in.ambient_kind != RQ_AMBIENT_CONSTANT && in.ambient_kind != RQ_AMBIENT_EYE)
    return false;
  if (in.background_kind != RQ_BACKGROUND_CONSTANT &&
      in.background_kind != RQ_BACKGROUND_LINEAR)
    return false;
  out.ambient_kind = in.ambient_kind == RQ_AMBIENT_EYE ? kAmbientEye : kAmbientConstant;
  out.background_kind =
      in.background_kind == RQ_BACKGROUND_LINEAR ? kBackgroundLinear : kBackgroundConstant;
  if (out.background_kind == kBackgroundLinear) {
    // LinearBackground's constructor: up.normalize() (VectorT::normalize)
    float up[3] = {in.background_up[0], in.background_up[1], in.background_up[2]};
    hnormalize(up);
    for (int c = 0; c < 3; ++c) {
      if (!std::isfinite(up[c])) return false;
      out.up[c] = up[c];
      out.down[c] = in.background_down[c];
    }
  }
  return true;
}

// Scratch of the frame path, owned by the scene and grown on demand.
struct FrameScratch {
  int32_t* counters = nullptr;
  unsigned long long* shadow = nullptr;
  float* materials = nullptr;
  int n_materials = 0;
  std::vector<float> host_materials;
  // host-output staging
  size_t out_npix = 0;
  float* d_rgb = nullptr;
  float* d_t = nullptr;
  int32_t* d_prim = nullptr;
  cudaStream_t stream = nullptr;
  ~FrameScratch() {
    cudaFree(counters);
    cudaFree(shadow);
    cudaFree(materials);
    cudaFree(d_rgb);
    cudaFree(d_t);
    cudaFree(d_prim);
    if (stream) cudaStreamDestroy(stream);
  }
};

void destroy_frame(FrameScratch* f) { delete f; }

static int set_fail(int code, const std::string& m) {
  set_error(m);
  return code;
}

static int prepare(Scene* s, const rq_whitted_params* p, FrameParams& P) {
  if (!p) return set_fail(RQ_ERR_ARG, "NULL params");
  if (p->xres <= 0 || p->yres <= 0 || (long long)p->xres * p->yres > (1LL << 30))
    return set_fail(RQ_ERR_ARG, "bad resolution");
  if (p->n_lights < 0 || p->n_lights > kMaxLights || (p->n_lights > 0 && !p->lights))
    return set_fail(RQ_ERR_ARG, "0..16 point lights");
  if (p->n_materials <= 0 || !p->material_rgb) return set_fail(RQ_ERR_ARG, "no materials");
  if (s->max_face_material >= p->n_materials)
    return set_fail(RQ_ERR_ARG, "face_material refers past n_materials");
  if (!s->has_tree) return set_fail(RQ_ERR_STATE, "scene has no tree");
  if (s->instanced) return set_fail(RQ_ERR_ARG, "instanced scene: render it with rq_render_frame");
  std::memset(&P, 0, sizeof(P));
  camera_basis(p->eye, p->lookat, p->up, p->hfov, p->vfov, P.cam);
  P.xres = p->xres;
  P.yres = p->yres;
  P.n_lights = p->n_lights;
  std::memcpy(P.lights, p->lights, sizeof(float) * 6 * p->n_lights);
  std::memcpy(P.ambient, p->ambient, sizeof(P.ambient));
  std::memcpy(P.background, p->background, sizeof(P.background));
  if (!environment_from(p->environment, P.env))
    return set_fail(RQ_ERR_ARG, "bad environment (kind, or a zero background up)");
  if (!s->frame) s->frame = new FrameScratch();
  FrameScratch* f = s->frame;
  if (!f->counters) {
    if (cudaMalloc(&f->counters, kNumCounters * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&f->shadow, sizeof(unsigned long long)) != cudaSuccess)
      return set_fail(RQ_ERR_OOM, "frame counters allocation failed");
  }
  const float* mrgb = p->material_rgb;
  if (f->n_materials != p->n_materials ||
      std::memcmp(f->host_materials.data(), mrgb, sizeof(float) * 3 * p->n_materials) != 0) {
    cudaFree(f->materials);
    f->materials = nullptr;
    if (cudaMalloc(&f->materials, sizeof(float) * 3 * p->n_materials) != cudaSuccess)
      return set_fail(RQ_ERR_OOM, "materials allocation failed");
    if (cudaMemcpy(f->materials, mrgb, sizeof(float) * 3 * p->n_materials,
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return set_fail(RQ_ERR_CUDA, "materials upload failed");
    f->host_materials.assign(mrgb, mrgb + 3 * p->n_materials);
    f->n_materials = p->n_materials;
  }
  P.materials = f->materials;
  return RQ_OK;
}

static int launch(Scene* s, const FrameParams& P, float* rgb, float* t, int32_t* prim,
                  unsigned long long* shadow, cudaStream_t st) {
  FrameScratch* f = s->frame;
  FrameBuffers B;
  B.rgb = rgb;
  B.t = t;
  B.prim = prim;
  B.counters = f->counters;
  B.shadow_rays_ptr = shadow ? shadow : f->shadow;
  B.stats = s->stats;
  const DevScene S = s->dev();
  const size_t smem = (size_t)S.depth * 128 * sizeof(int2);
  const int bps = whitted_blocks_per_sm(s->tri_kind, smem);
  const int npix = P.xres * P.yres;
  const int grid = std::max(1, std::min(bps * s->num_sms, (npix + 127) / 128));
  cudaError_t e = launch_whitted(S, P, B, grid, st, s->stage_events, s->n_stage_events);
  if (e != cudaSuccess) return set_fail(RQ_ERR_CUDA, std::string("whitted launch: ") +
                                                         cudaGetErrorString(e));
  return RQ_OK;
}

}  // namespace rq

extern "C" {

int rq_camera_basis(const float* eye, const float* lookat, const float* up, float hfov,
                    float vfov, float* out12) {
  if (!eye || !lookat || !up || !out12) return rq::set_fail(RQ_ERR_ARG, "NULL argument");
  rq::camera_basis(eye, lookat, up, hfov, vfov, out12);
  return RQ_OK;
}

int rq_render_whitted_device(rq_scene* scene, const rq_whitted_params* params, float* d_rgb,
                             float* d_t, int32_t* d_prim, uint64_t* d_shadow_rays,
                             void* stream) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s || !d_rgb || !d_t || !d_prim) return rq::set_fail(RQ_ERR_ARG, "NULL argument");
  if (cudaSetDevice(s->device) != cudaSuccess) return rq::set_fail(RQ_ERR_CUDA, "cudaSetDevice");
  std::lock_guard<std::mutex> g(s->frame_mu);
  rq::FrameParams P;
  int rc = rq::prepare(s, params, P);
  if (rc != RQ_OK) return rc;
  return rq::launch(s, P, d_rgb, d_t, d_prim,
                    reinterpret_cast<unsigned long long*>(d_shadow_rays),
                    static_cast<cudaStream_t>(stream));
}

int rq_render_whitted(rq_scene* scene, const rq_whitted_params* params, float* rgb, float* t,
                      int32_t* prim, uint64_t* shadow_rays) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s || !rgb) return rq::set_fail(RQ_ERR_ARG, "NULL argument");
  if (cudaSetDevice(s->device) != cudaSuccess) return rq::set_fail(RQ_ERR_CUDA, "cudaSetDevice");
  std::lock_guard<std::mutex> g(s->frame_mu);
  rq::FrameParams P;
  int rc = rq::prepare(s, params, P);
  if (rc != RQ_OK) return rc;
  rq::FrameScratch* f = s->frame;
  const size_t npix = (size_t)params->xres * params->yres;
  if (!f->stream && cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking) != cudaSuccess)
    return rq::set_fail(RQ_ERR_CUDA, "stream creation failed");
  if (f->out_npix < npix) {
    cudaFree(f->d_rgb);
    cudaFree(f->d_t);
    cudaFree(f->d_prim);
    f->d_rgb = f->d_t = nullptr;
    f->d_prim = nullptr;
    if (cudaMalloc(&f->d_rgb, npix * 12) != cudaSuccess ||
        cudaMalloc(&f->d_t, npix * 4) != cudaSuccess ||
        cudaMalloc(&f->d_prim, npix * 4) != cudaSuccess)
      return rq::set_fail(RQ_ERR_OOM, "frame output allocation failed");
    f->out_npix = npix;
  }
  rc = rq::launch(s, P, f->d_rgb, f->d_t, f->d_prim, nullptr, f->stream);
  if (rc != RQ_OK) return rc;
  cudaError_t e = cudaMemcpyAsync(rgb, f->d_rgb, npix * 12, cudaMemcpyDeviceToHost, f->stream);
  if (e == cudaSuccess && t) e = cudaMemcpyAsync(t, f->d_t, npix * 4, cudaMemcpyDeviceToHost, f->stream);
  if (e == cudaSuccess && prim)
    e = cudaMemcpyAsync(prim, f->d_prim, npix * 4, cudaMemcpyDeviceToHost, f->stream);
  unsigned long long ns = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&ns, f->shadow, sizeof(ns), cudaMemcpyDeviceToHost, f->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) return rq::set_fail(RQ_ERR_CUDA, std::string("frame copy: ") + cudaGetErrorString(e));
  if (shadow_rays) *shadow_rays = ns;
  return RQ_OK;
}

}  // extern "C"
