// Host entry points of the path-tracing wavefront (rq_render_path*).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_path.h"
#include "rq_render.h"
#include "rq_scene.h"

namespace rq {

struct PathScratch {
  size_t capacity = 0;
  PathBuffers B{};
  float* materials = nullptr;
  std::vector<float> host_materials;
  unsigned long long* counts = nullptr;  // default ray counters
  float* d_rgb = nullptr;
  size_t rgb_pix = 0;
  cudaStream_t stream = nullptr;
  void free_paths() {
    cudaFree(B.o); cudaFree(B.d); cudaFree(B.imp); cudaFree(B.rad); cudaFree(B.rng);
    cudaFree(B.t); cudaFree(B.pos); cudaFree(B.prim); cudaFree(B.queue[0]);
    cudaFree(B.queue[1]); cudaFree(B.counters); cudaFree(B.alive); cudaFree(B.tile_counts);
    B.o = B.d = B.imp = B.rad = B.t = nullptr;
    B.rng = nullptr;
    B.alive = nullptr;
    B.pos = B.prim = B.queue[0] = B.queue[1] = B.counters = B.tile_counts = nullptr;
    capacity = 0;
  }
  ~PathScratch() {
    free_paths();
    cudaFree(materials);
    cudaFree(counts);
    cudaFree(d_rgb);
    if (stream) cudaStreamDestroy(stream);
  }
};

void destroy_path_scratch(PathScratch* p) { delete p; }

static int pfail(int code, const std::string& m) {
  set_error(m);
  return code;
}

template <class T>
static bool palloc(T** p, size_t n) {
  return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess;
}

static int path_prepare(Scene* s, const rq_path_params* p, PathParams& P, long long& total,
                        int& chunk) {
  if (!p) return pfail(RQ_ERR_ARG, "NULL params");
  if (p->xres <= 0 || p->yres <= 0) return pfail(RQ_ERR_ARG, "bad resolution");
  const int strata = (int)std::lround(std::sqrt((double)p->spp));
  if (p->spp <= 0 || strata * strata != p->spp || p->spp > 4096)
    return pfail(RQ_ERR_ARG, "spp must be a perfect square (1, 4, 16, ...)");
  if (p->max_depth < 1 || p->max_depth > kMaxPathDepth)
    return pfail(RQ_ERR_ARG, "max_depth must be in [1, 16]");
  if (p->n_materials <= 0 || !p->material_rgb) return pfail(RQ_ERR_ARG, "no materials");
  if (s->max_face_material >= p->n_materials)
    return pfail(RQ_ERR_ARG, "face_material past n_materials");
  if (!s->has_tree) return pfail(RQ_ERR_STATE, "scene has no tree");
  if (s->instanced) return pfail(RQ_ERR_ARG, "path tracing takes triangle scenes");
  std::memset(&P, 0, sizeof(P));
  camera_basis(p->eye, p->lookat, p->up, p->hfov, p->vfov, P.cam);
  P.xres = p->xres;
  P.yres = p->yres;
  P.spp = p->spp;
  P.strata = strata;
  P.max_depth = p->max_depth;
  P.rr_depth = p->rr_depth;
  P.seed = p->seed;
  for (int c = 0; c < 3; ++c) {
    P.light_anchor[c] = p->light_anchor[c];
    P.light_v1[c] = p->light_v1[c];
    P.light_v2[c] = p->light_v2[c];
    P.light_color[c] = p->light_color[c];
    P.background[c] = p->background[c];
    P.ambient[c] = p->ambient[c];
  }
  if (!environment_from(p->environment, P.env))
    return pfail(RQ_ERR_ARG, "bad environment (kind, or a zero background up)");
  // Parallelogram constructor (Model/Primitives/Parallelogram.cc:26-35)
  float n[3] = {p->light_v1[1] * p->light_v2[2] - p->light_v1[2] * p->light_v2[1],
                p->light_v1[2] * p->light_v2[0] - p->light_v1[0] * p->light_v2[2],
                p->light_v1[0] * p->light_v2[1] - p->light_v1[1] * p->light_v2[0]};
  const float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  const float sc = 1 / l;
  for (int c = 0; c < 3; ++c) P.light_normal[c] = n[c] * sc;
  P.light_inv_area = (float)1 / l;
  total = (long long)p->xres * p->yres * p->spp;
  long long ch = p->chunk_paths > 0 ? p->chunk_paths : (4LL << 20);
  ch = std::max<long long>(ch / p->spp, 1) * p->spp;  // whole pixels per chunk
  chunk = (int)std::min<long long>(ch, total);
  if (!s->paths) s->paths = new PathScratch();
  PathScratch* ps = s->paths;
  if (ps->capacity < (size_t)chunk) {
    ps->free_paths();
    const size_t C = (size_t)chunk;
    PathBuffers& B = ps->B;
    if (!palloc(&B.o, 3 * C) || !palloc(&B.d, 3 * C) || !palloc(&B.imp, 3 * C) ||
        !palloc(&B.rad, 3 * C) || !palloc(&B.rng, C) || !palloc(&B.t, C) ||
        !palloc(&B.pos, C) || !palloc(&B.prim, C) || !palloc(&B.queue[0], C) ||
        !palloc(&B.queue[1], C) || !palloc(&B.counters, kPathCounters) ||
        !palloc(&B.alive, C) || !palloc(&B.tile_counts, C / 4096 + 2)) {
      ps->free_paths();
      return pfail(RQ_ERR_OOM, "path state allocation failed");
    }
    ps->capacity = C;
    B.capacity = C;
  }
  if (!ps->counts && !palloc(&ps->counts, 2)) return pfail(RQ_ERR_OOM, "counter allocation");
  const float* mrgb = p->material_rgb;
  if ((int)ps->host_materials.size() != 3 * p->n_materials ||
      std::memcmp(ps->host_materials.data(), mrgb, sizeof(float) * 3 * p->n_materials) != 0) {
    cudaFree(ps->materials);
    ps->materials = nullptr;
    if (!palloc(&ps->materials, 3 * (size_t)p->n_materials) ||
        cudaMemcpy(ps->materials, mrgb, sizeof(float) * 3 * p->n_materials,
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return pfail(RQ_ERR_OOM, "materials upload failed");
    ps->host_materials.assign(mrgb, mrgb + 3 * p->n_materials);
  }
  P.materials = ps->materials;
  return RQ_OK;
}

static int path_run(Scene* s, const PathParams& P, long long total, int chunk, float* d_rgb,
                    unsigned long long* d_counts, cudaStream_t st) {
  PathScratch* ps = s->paths;
  PathBuffers B = ps->B;
  B.ray_counts = d_counts ? d_counts : ps->counts;
  B.stats = s->stats;
  B.dbg_prim = s->path_dbg_prim;
  B.dbg_org = s->path_dbg_org;
  B.dbg_dir = s->path_dbg_dir;
  if (B.dbg_prim && (long long)s->path_dbg_capacity < total)
    return pfail(RQ_ERR_ARG, "debug buffers smaller than the frame's path count");
  if (B.dbg_prim && chunk != total) return pfail(RQ_ERR_ARG, "debug dump needs a single chunk");
  DevScene S;
  int lrc = s->node_layout(s->cfg[RQ_PATH_EXTEND].node_layout, S);
  if (lrc != RQ_OK) return lrc;
  const size_t smem = (size_t)S.depth * 128 * sizeof(int2);
  const int grid = std::max(1, path_blocks_per_sm(s->tri_kind, smem) * s->num_sms);
  PathLaunch L;
  for (int k = 0; k < 2; ++k) {
    const rq_launch_config& c = s->cfg[RQ_PATH_EXTEND + k];
    L.block_threads[k] = c.block_threads;
    L.blocks_per_sm[k] = c.blocks_per_sm;
    L.refill[k] = c.refill_threshold;
    L.reg_stack[k] = c.reg_stack;
  }
  cudaError_t e = cudaMemsetAsync(B.ray_counts, 0, 2 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return pfail(RQ_ERR_CUDA, cudaGetErrorString(e));
  for (long long g0 = 0; g0 < total; g0 += chunk) {
    const int n = (int)std::min<long long>(chunk, total - g0);
    e = launch_path_chunk(S, P, B, g0, n, d_rgb, grid, L, st, s->stage_events,
                          s->n_stage_events);
    if (e != cudaSuccess) return pfail(RQ_ERR_CUDA, std::string("path launch: ") + cudaGetErrorString(e));
  }
  return RQ_OK;
}

}  // namespace rq

extern "C" {

int rq_render_path_device(rq_scene* scene, const rq_path_params* params, float* d_rgb,
                          uint64_t* d_ray_counts, void* stream) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s || !d_rgb) return rq::pfail(RQ_ERR_ARG, "NULL argument");
  if (cudaSetDevice(s->device) != cudaSuccess) return rq::pfail(RQ_ERR_CUDA, "cudaSetDevice");
  std::lock_guard<std::mutex> g(s->frame_mu);
  rq::PathParams P;
  long long total;
  int chunk;
  int rc = rq::path_prepare(s, params, P, total, chunk);
  if (rc != RQ_OK) return rc;
  return rq::path_run(s, P, total, chunk, d_rgb,
                      reinterpret_cast<unsigned long long*>(d_ray_counts),
                      static_cast<cudaStream_t>(stream));
}

int rq_render_path(rq_scene* scene, const rq_path_params* params, float* rgb,
                   uint64_t* ray_counts) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s || !rgb) return rq::pfail(RQ_ERR_ARG, "NULL argument");
  if (cudaSetDevice(s->device) != cudaSuccess) return rq::pfail(RQ_ERR_CUDA, "cudaSetDevice");
  std::lock_guard<std::mutex> g(s->frame_mu);
  rq::PathParams P;
  long long total;
  int chunk;
  int rc = rq::path_prepare(s, params, P, total, chunk);
  if (rc != RQ_OK) return rc;
  rq::PathScratch* ps = s->paths;
  const size_t npix = (size_t)params->xres * params->yres;
  if (!ps->stream && cudaStreamCreateWithFlags(&ps->stream, cudaStreamNonBlocking) != cudaSuccess)
    return rq::pfail(RQ_ERR_CUDA, "stream creation failed");
  if (ps->rgb_pix < npix) {
    cudaFree(ps->d_rgb);
    ps->d_rgb = nullptr;
    if (!rq::palloc(&ps->d_rgb, 3 * npix)) return rq::pfail(RQ_ERR_OOM, "image allocation");
    ps->rgb_pix = npix;
  }
  rc = rq::path_run(s, P, total, chunk, ps->d_rgb, nullptr, ps->stream);
  if (rc != RQ_OK) return rc;
  unsigned long long counts[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(rgb, ps->d_rgb, 12 * npix, cudaMemcpyDeviceToHost, ps->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(counts, ps->counts, sizeof(counts), cudaMemcpyDeviceToHost, ps->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ps->stream);
  if (e != cudaSuccess) return rq::pfail(RQ_ERR_CUDA, cudaGetErrorString(e));
  if (ray_counts) {
    ray_counts[0] = counts[0];
    ray_counts[1] = counts[1];
  }
  return RQ_OK;
}

int rq_set_path_debug(rq_scene* scene, int32_t* d_prim, float* d_org, float* d_dir,
                      int64_t capacity_paths) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s) return rq::pfail(RQ_ERR_ARG, "NULL scene");
  if (d_prim && (!d_org || !d_dir || capacity_paths <= 0))
    return rq::pfail(RQ_ERR_ARG, "debug dump needs prim, org and dir buffers");
  s->path_dbg_prim = d_prim;
  s->path_dbg_org = d_org;
  s->path_dbg_dir = d_dir;
  s->path_dbg_capacity = d_prim ? capacity_paths : 0;
  return RQ_OK;
}

}  // extern "C"
