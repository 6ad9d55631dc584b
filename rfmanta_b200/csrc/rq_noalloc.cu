// rq_render_whitted_device_noalloc: the Whitted frame of
// rq_render_whitted_device for callers that must not allocate device memory,
// e.g. a render worker whose process has handed all of HBM to another
// allocator, or a host thread that may not call cudaMalloc/cudaFree because
// those calls can synchronise the device in the middle of its work.
//
// The frame's scratch - the work counters, the shadow-ray counter and the
// material table - lives in one file-scope __device__ array of fixed size
// instead of buffers the scene allocates on first use.  The frame kernel
// keeps no per-pixel scratch, so any resolution the allocating entry point
// takes is accepted; the limit is kNoAllocMaxMaterials materials per frame.
//
// Host code cannot use the array's name as a device address (on the host it
// names a host-side stand-in).  The device address is looked up with
// cudaGetSymbolAddress once per device, with that device current, on the
// first call made for that device, and cached.
//
// Every call on a device shares the one array and the array keeps the last
// call's contents: the counters are cleared at the start of every frame, and
// two calls whose work overlaps on the GPU (different streams, no ordering)
// race on the array.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/rfmanta_b200.h"
#include "rq_render.h"
#include "rq_scene.h"

namespace rq {

constexpr int kNoAllocMaxMaterials = 1024;

// Byte offsets inside the array (each region 256-byte aligned).
constexpr size_t kOffCounters = 0;
constexpr size_t kOffShadow = kOffCounters + 256;
constexpr size_t kOffMaterials = kOffShadow + 256;
constexpr size_t kNoAllocBytes = kOffMaterials + 12 * (size_t)kNoAllocMaxMaterials;

static __device__ __align__(256) unsigned char g_frame_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
static void* g_scratch_addr[kNoAllocMaxDevices] = {};
static std::mutex g_scratch_mu;

static int na_fail(int code, const std::string& m) {
  set_error(m);
  return code;
}

// Device address of g_frame_scratch on the current device `device`.
static int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kNoAllocMaxDevices)
    return na_fail(RQ_ERR_ARG, "device ordinal beyond the no-alloc table");
  std::lock_guard<std::mutex> g(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_frame_scratch);
    if (e != cudaSuccess || !p)
      return na_fail(RQ_ERR_CUDA, std::string("cudaGetSymbolAddress(frame scratch): ") +
                                      cudaGetErrorString(e));
    g_scratch_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[device]);
  return RQ_OK;
}

}  // namespace rq

extern "C" int rq_render_whitted_device_noalloc(rq_scene* scene,
                                                const rq_whitted_params* p, float* d_rgb,
                                                float* d_t, int32_t* d_prim,
                                                uint64_t* d_shadow_rays, void* stream) {
  using namespace rq;
  Scene* s = reinterpret_cast<Scene*>(scene);
  if (!s || !p || !d_rgb || !d_t || !d_prim) return na_fail(RQ_ERR_ARG, "NULL argument");
  if (p->xres <= 0 || p->yres <= 0) return na_fail(RQ_ERR_ARG, "bad resolution");
  const size_t npix = (size_t)p->xres * (size_t)p->yres;
  if (npix > (size_t(1) << 30)) return na_fail(RQ_ERR_ARG, "bad resolution");
  if (p->n_materials <= 0 || !p->material_rgb) return na_fail(RQ_ERR_ARG, "no materials");
  if (p->n_materials > kNoAllocMaxMaterials)
    return na_fail(RQ_ERR_CAPACITY,
                   "rq_render_whitted_device_noalloc: more than " +
                       std::to_string(kNoAllocMaxMaterials) + " materials");
  if (p->n_lights < 0 || p->n_lights > kMaxLights || (p->n_lights > 0 && !p->lights))
    return na_fail(RQ_ERR_ARG, "0..16 point lights");
  if (s->instanced) return na_fail(RQ_ERR_ARG, "instanced scene: render it with rq_render_frame");
  if (cudaSetDevice(s->device) != cudaSuccess) return na_fail(RQ_ERR_CUDA, "cudaSetDevice");
  // The scene's tree, statistics pointer and material maximum may be
  // replaced by an update on another host thread (an update can free and
  // reallocate the node records); the same per-scene lock as the allocating
  // entry point keeps this frame's snapshot of them valid.  A host mutex
  // makes no device call.
  std::lock_guard<std::mutex> g(s->frame_mu);
  if (s->max_face_material >= p->n_materials)
    return na_fail(RQ_ERR_ARG, "face_material past n_materials");
  if (!s->has_tree) return na_fail(RQ_ERR_STATE, "scene has no tree");
  unsigned char* base = nullptr;
  int rc = scratch_address(s->device, &base);
  if (rc != RQ_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  FrameParams P;
  std::memset(&P, 0, sizeof(P));
  camera_basis(p->eye, p->lookat, p->up, p->hfov, p->vfov, P.cam);
  P.xres = p->xres;
  P.yres = p->yres;
  P.n_lights = p->n_lights;
  std::memcpy(P.lights, p->lights, sizeof(float) * 6 * p->n_lights);
  std::memcpy(P.ambient, p->ambient, sizeof(P.ambient));
  std::memcpy(P.background, p->background, sizeof(P.background));
  if (!environment_from(p->environment, P.env))
    return na_fail(RQ_ERR_ARG, "bad environment (kind, or a zero background up)");
  float* mats = reinterpret_cast<float*>(base + kOffMaterials);
  // cudaMemcpyDefault: the table may sit in pinned host memory (an
  // asynchronous copy) or in device memory; a pageable host table is
  // accepted too, but the driver then stages it and the call may block.
  cudaError_t e = cudaMemcpyAsync(mats, p->material_rgb, sizeof(float) * 3 * p->n_materials,
                                  cudaMemcpyDefault, st);
  if (e != cudaSuccess) return na_fail(RQ_ERR_CUDA, std::string("materials: ") + cudaGetErrorString(e));
  P.materials = mats;

  FrameBuffers B;
  B.rgb = d_rgb;
  B.t = d_t;
  B.prim = d_prim;
  B.counters = reinterpret_cast<int32_t*>(base + kOffCounters);
  B.shadow_rays_ptr = d_shadow_rays ? reinterpret_cast<unsigned long long*>(d_shadow_rays)
                                    : reinterpret_cast<unsigned long long*>(base + kOffShadow);
  B.stats = s->stats;
  const DevScene S = s->dev();
  const size_t smem = (size_t)S.depth * 128 * sizeof(int2);
  const int grid = std::max(1, std::min(whitted_blocks_per_sm(s->tri_kind, smem) * s->num_sms,
                                        (int)((npix + 127) / 128)));
  // launch_whitted clears the work counters and the shadow counter first
  e = launch_whitted(S, P, B, grid, st, nullptr, 0);
  if (e != cudaSuccess) return na_fail(RQ_ERR_CUDA, std::string("whitted launch: ") + cudaGetErrorString(e));
  return RQ_OK;
}
