// Served path tracing with continuous batching (rq_server_*).
//
// Device side: one wavefront step serves chunks of many requests at once.
// A chunk is a fixed range of whole pixels of one request (all of their
// samples); each path slot of the step's pool records its request and its
// global path id inside that request, and every kernel reads the slot's own
// request parameters and scene.  A path's computation depends only on
// (request, path id) - its PCG32 stream, camera sample, scene and depth -
// and every pixel is resolved inside the chunk that holds all its samples,
// so a request's image is the same bits whether it ran alone or mixed with
// any other requests.
//
// Host side (the engine): requests are queued on submit, admitted in
// arrival order while their output image fits the HBM budget, and each
// step gives every admitted request one chunk, then fills the rest of the
// path pool oldest request first; at most two steps are in flight, and a
// request completes when the step holding its last chunk has finished on the
// device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_batch.h"
#include "rq_pathcore.cuh"
#include "rq_render.h"
#include "rq_scene.h"

namespace rq {

constexpr int kMaxServeScenes = 32;

struct ServeReq {
  PathParams P;
  int scene;
  float* out;  // device rgb image
};

struct ServeChunk {
  int req;    // index into the step's request table
  int pix0;   // first pixel of the chunk in the request's image
  int npix;
  int slot0;  // first path slot of the chunk in the pool
  int px0;    // prefix of pixels over the step's chunks
};

struct ServeArgs {
  const DevScene* scenes;
  int n_scenes;
  const ServeReq* reqs;
  const ServeChunk* chunks;
  int n_chunks;
  int n_slots;  // paths in this step
  int n_pix;    // pixels in this step
  int* slot_req;
  long long* slot_g;
};

__device__ __forceinline__ int find_chunk_by_slot(const ServeArgs& A, int s) {
  int lo = 0, hi = A.n_chunks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (A.chunks[mid].slot0 <= s) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void serve_generate_kernel(ServeArgs A, PathBuffers B) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < A.n_slots;
       s += gridDim.x * blockDim.x) {
    const ServeChunk c = A.chunks[find_chunk_by_slot(A, s)];
    const ServeReq& R = A.reqs[c.req];
    const long long g = (long long)c.pix0 * R.P.spp + (s - c.slot0);
    generate_path(R.P, B, g, s);
    A.slot_req[s] = c.req;
    A.slot_g[s] = g;
  }
}

__device__ __forceinline__ void stage_scenes(const ServeArgs& A, DevScene* sm) {
  for (int i = threadIdx.x; i < A.n_scenes; i += blockDim.x) sm[i] = A.scenes[i];
  __syncthreads();
}

// Lanes that must be idle before a warp of the persistent stages fetches
// new path slots (the path tracer's tuned defaults).
constexpr int kServeExtendRefill = 16;
constexpr int kServeShadeRefill = 24;

// Persistent extension stage over the step's live slots: each lane keeps one
// slot's ray in flight in that slot's request scene; warps refill idle lanes
// with one atomic on the bounce's work counter (as path_extend_persistent_
// kernel does for a single frame).
template <int KIND>
__global__ void __launch_bounds__(128) serve_extend_kernel(ServeArgs A, PathBuffers B, int depth) {
  extern __shared__ int2 smem_stack[];
  __shared__ DevScene sm_scenes[kMaxServeScenes];
  stage_scenes(A, sm_scenes);
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  const int nq = depth == 0 ? A.n_slots : *(volatile const int*)&B.counters[depth];
  const int* qin = B.queue[depth & 1];
  int* counter = &B.counters[kFetchBase + depth];
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  int p = -1, scene = 0;
  const ServeReq* R = nullptr;
  bool exhausted = false;
  Ray r;
  Hit h;
  int ref = kDone, sp = 0;
  for (;;) {
    const bool idle = (p < 0) && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, idle);
    const unsigned busy = __ballot_sync(0xffffffffu, p >= 0);
    if (m != 0u && (__popc(m) >= kServeExtendRefill || busy == 0u)) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (idle) {
        const int qi = base + __popc(m & lt_mask);
        if (qi < nq) {
          p = depth == 0 ? qi : qin[qi];
          R = &A.reqs[A.slot_req[p]];
          scene = R->scene;
          load_extension_ray(B, p, r);
          start_ray(sm_scenes[scene], r, h, ref, sp);
        } else {
          exhausted = true;
        }
      }
    }
    if (__all_sync(0xffffffffu, exhausted)) break;
    if (p >= 0) {
      if (ref != kDone) {
        // scene pointers in registers: the stack stores would otherwise make
        // every node visit read them from shared memory again
        DevScene S;
        S.nodes = sm_scenes[scene].nodes;
        S.tris = sm_scenes[scene].tris;
        step<KIND, false>(S, r, h, ref, sp, stk, stride);
      }
      if (ref == kDone) {
        store_extension(R->P, B, depth, p, r, h);
        p = -1;
      }
    }
  }
}

// Persistent shade stage: shade_begin, the shadow ray's any-hit steps and
// shade_finish per lane, survivors compacted into the next queue at the
// warp's common point.
template <int KIND>
__global__ void __launch_bounds__(128) serve_shade_kernel(ServeArgs A, PathBuffers B, int depth) {
  extern __shared__ int2 smem_stack[];
  __shared__ DevScene sm_scenes[kMaxServeScenes];
  stage_scenes(A, sm_scenes);
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  const int nq = depth == 0 ? A.n_slots : *(volatile const int*)&B.counters[depth];
  const int* qin = B.queue[depth & 1];
  int* qout = B.queue[(depth + 1) & 1];
  int* counter = &B.counters[kShadeFetchBase + depth];
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  int p = -1, scene = 0, nshadow = 0;
  bool exhausted = false, alive = false, traced = false;
  float contrib[3];
  Ray sr;
  Hit sh;
  int ref = kDone, sp = 0;
  for (;;) {
    const bool idle = (p < 0) && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, idle);
    const unsigned busy = __ballot_sync(0xffffffffu, p >= 0);
    if (m != 0u && (__popc(m) >= kServeShadeRefill || busy == 0u)) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (idle) {
        const int qi = base + __popc(m & lt_mask);
        if (qi < nq) {
          p = depth == 0 ? qi : qin[qi];
          const ServeReq& R = A.reqs[A.slot_req[p]];
          scene = R.scene;
          // a request whose depth is already reached keeps no live paths here
          traced = shade_begin<KIND>(sm_scenes[scene], R.P, B, depth, p, A.slot_g[p], sr,
                                     contrib, alive);
          ref = kDone;
          if (traced) {
            ++nshadow;
            start_ray(sm_scenes[scene], sr, sh, ref, sp);
          }
        } else {
          exhausted = true;
        }
      }
    }
    if (__all_sync(0xffffffffu, exhausted)) break;
    bool fin = false;
    if (p >= 0) {
      if (ref != kDone) {
        DevScene S;
        S.nodes = sm_scenes[scene].nodes;
        S.tris = sm_scenes[scene].tris;
        step<KIND, true>(S, sr, sh, ref, sp, stk, stride);
      }
      if (ref == kDone) {
        if (traced && sh.id < 0) shade_finish(B, p, contrib);
        fin = true;
      }
    }
    if (B.alive) {  // survivors are compacted in slot order after the kernel
      if (fin) {
        B.alive[p] = alive ? 1 : 0;
        p = -1;
      }
      continue;
    }
    const bool push = fin && alive;
    const unsigned pm = __ballot_sync(0xffffffffu, push);
    if (pm) {
      const int leader = __ffs(pm) - 1;
      int q = 0;
      if ((int)lane == leader) q = atomicAdd(&B.counters[depth + 1], __popc(pm));
      q = __shfl_sync(0xffffffffu, q, leader);
      if (push) qout[q + __popc(pm & lt_mask)] = p;
    }
    if (fin) p = -1;
  }
  int tot = nshadow;
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
  if (lane == 0 && tot) atomicAdd(&B.ray_counts[1], (unsigned long long)tot);
}

__global__ void serve_count_kernel(ServeArgs A, PathBuffers B, int depth) {
  if (threadIdx.x == 0 && blockIdx.x == 0)
    atomicAdd(&B.ray_counts[0],
              (unsigned long long)(depth == 0 ? A.n_slots : B.counters[depth]));
}

// Per pixel of the step: the mean of its samples in sample order, written
// into the request's image.
__global__ void serve_resolve_kernel(ServeArgs A, PathBuffers B) {
  const size_t C = B.capacity;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < A.n_pix; k += gridDim.x * blockDim.x) {
    int lo = 0, hi = A.n_chunks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (A.chunks[mid].px0 <= k) lo = mid;
      else hi = mid - 1;
    }
    const ServeChunk c = A.chunks[lo];
    const ServeReq& R = A.reqs[c.req];
    const int j = k - c.px0;
    const int spp = R.P.spp;
    const float inv = fdiv(1.f, (float)spp);
    float acc[3] = {0.f, 0.f, 0.f};
    for (int s = 0; s < spp; ++s) {
      const int p = c.slot0 + j * spp + s;
#pragma unroll
      for (int q = 0; q < 3; ++q) acc[q] = fadd(acc[q], B.rad[q * C + p]);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) R.out[3 * (size_t)(c.pix0 + j) + q] = fmul(acc[q], inv);
  }
}

template <int KIND>
static cudaError_t serve_launch_step(const ServeArgs& A, PathBuffers B, int max_depth,
                                     int grid, size_t smem, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(B.counters, 0, kPathCounters * sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int gg = std::max(1, std::min(grid, (A.n_slots + 255) / 256));
  serve_generate_kernel<<<gg, 256, 0, st>>>(A, B);
  for (int depth = 0; depth < max_depth; ++depth) {
    serve_count_kernel<<<1, 32, 0, st>>>(A, B, depth);
    serve_extend_kernel<KIND><<<grid, 128, smem, st>>>(A, B, depth);
    cudaMemsetAsync(B.alive, 0, (size_t)A.n_slots, st);
    serve_shade_kernel<KIND><<<grid, 128, smem, st>>>(A, B, depth);
    launch_ordered_compaction(B, A.n_slots, depth, st);
  }
  const int rg = std::max(1, std::min(grid, (A.n_pix + 255) / 256));
  serve_resolve_kernel<<<rg, 256, 0, st>>>(A, B);
  return cudaGetLastError();
}

static int serve_blocks_per_sm(int kind, size_t smem) {
  const void* fs[2] = {kind == kWald ? (const void*)serve_extend_kernel<kWald>
                                     : (const void*)serve_extend_kernel<kKS>,
                       kind == kWald ? (const void*)serve_shade_kernel<kWald>
                                     : (const void*)serve_shade_kernel<kKS>};
  int a = 1, b = 1;
  for (const void* f : fs)
    if (smem > 0)  // the static scene table counts against the default 48 KB too
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, fs[0], 128, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fs[1], 128, smem);
  return std::max(1, std::min(a, b));
}

}  // namespace rq

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int sfail(int code, const std::string& m) {
  rq::set_error(m);
  return code;
}

struct HostReq {
  int id = 0;
  // a ray-query request: n_rays rays of one scene, closest or any hit,
  // copied to the device on admission and traced in chunks of the steps
  bool query = false;
  int n_rays = 0;
  int flags = 0;
  std::vector<float> rays;    // host copy: org 3n, dir 3n, tmax n
  float* d_rays = nullptr;    // the same on the device
  float* d_res = nullptr;     // t n, prim n
  int next_ray = 0;
  rq_serve_request spec{};
  std::vector<float> materials;
  rq::ServeReq dev{};  // parameters as the kernels see them (out, materials set on admission)
  float* d_mat = nullptr;
  float* d_out = nullptr;
  size_t bytes = 0;
  int npix = 0;
  int next_pix = 0;
  bool admitted = false;
  bool scheduled_all = false;
  bool done = false;
  bool reported = false;
  cudaEvent_t done_ev = nullptr;
  double t_submit = 0, t_admit = 0, t_done = 0;
};

}  // namespace

struct rq_server {
  int device = 0;
  int tri_kind = 0;
  int num_sms = 148;
  std::vector<rq::Scene*> scenes;
  rq::DevScene* d_scenes = nullptr;
  int n_scenes = 0;
  int depth = 1;
  long long capacity = 0;
  int chunk_pixels = 0;
  size_t budget = 0;
  size_t used = 0;
  int max_active = 256;
  int max_chunks = 8192;
  rq::PathBuffers B{};
  int* slot_req = nullptr;
  long long* slot_g = nullptr;
  unsigned long long* counts = nullptr;
  rq::ServeReq* d_reqs = nullptr;
  rq::ServeChunk* d_chunks = nullptr;
  // pinned staging ring for the per-step tables
  static const int kRing = 3;
  rq::ServeReq* h_reqs[kRing] = {};
  rq::ServeChunk* h_chunks[kRing] = {};
  cudaEvent_t ring_ev[kRing] = {};   // after a step's table upload
  cudaEvent_t end_ev[kRing] = {};    // after a step's last kernel
  bool ring_used[kRing] = {};
  cudaStream_t stream = nullptr;
  // result copies wait for their request's completion event on a stream of
  // their own, so a copy never waits for steps enqueued after its request
  cudaStream_t copy_stream = nullptr;
  // request images come from the server's own memory pool, which keeps
  // what it has mapped (release threshold = all): the device's default
  // pool returns freed memory at every synchronisation, and mapping it
  // again stalls the request loop
  cudaMemPool_t pool = nullptr;
  std::map<int, std::unique_ptr<HostReq>> reqs;
  std::deque<int> pending;   // submitted, not admitted
  std::vector<int> active;   // admitted, not finished (admission order)
  std::vector<int> table;    // request id per device-table slot
  int next_id = 1;
  long long steps = 0;
  int grid = 1;
  size_t smem = 0;
  // the scenes' descriptors as uploaded and their generations: a scene
  // updated since (refit, rotations, new tree) gets its descriptor copied in
  // again before the next step
  std::vector<uint64_t> generations;
  std::vector<rq::DevScene> host_scenes;
  // ray-query chunks of a step: descriptors for the batched traversal
  // kernel (pinned staging per ring slot, one device table) and its counter
  static const int kMaxQueryDescs = 1024;
  rq::BatchDesc* h_qdesc[kRing] = {};
  rq::BatchDesc* d_qdesc = nullptr;
  int* d_qcounter = nullptr;
  int qgrid = 1;
  unsigned long long query_rays = 0;
  // per-step records (rq_server_set_profile): timing events around each
  // step's kernels, the record of the step in each ring slot until its end
  // event has been seen, finished records
  bool profile = false;
  double prof_t0 = 0;
  cudaEvent_t prof_start[kRing] = {};
  cudaEvent_t prof_end[kRing] = {};
  rq_server_step_record prof_slot[kRing] = {};
  bool prof_open[kRing] = {};
  std::vector<rq_server_step_record> prof_done;

  // Moves the record of ring slot `slot` to the finished list once its
  // end event has completed (blocking if `wait`).
  void close_profile(int slot, bool wait) {
    if (!prof_open[slot]) return;
    if (!wait && cudaEventQuery(prof_end[slot]) != cudaSuccess) return;
    if (wait) cudaEventSynchronize(prof_end[slot]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, prof_start[slot], prof_end[slot]);
    prof_slot[slot].gpu_ms = ms;
    prof_done.push_back(prof_slot[slot]);
    prof_open[slot] = false;
  }

  ~rq_server() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (auto& kv : reqs) {
      HostReq& r = *kv.second;
      if (r.d_out) cudaFreeAsync(r.d_out, stream);
      if (r.d_mat) cudaFreeAsync(r.d_mat, stream);
      if (r.d_rays) cudaFreeAsync(r.d_rays, stream);
      if (r.d_res) cudaFreeAsync(r.d_res, stream);
      if (r.done_ev) cudaEventDestroy(r.done_ev);
    }
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(d_qdesc);
    cudaFree(d_qcounter);
    for (int i = 0; i < kRing; ++i) cudaFreeHost(h_qdesc[i]);
    cudaFree(B.o); cudaFree(B.d); cudaFree(B.imp); cudaFree(B.rad); cudaFree(B.rng);
    cudaFree(B.t); cudaFree(B.pos); cudaFree(B.prim); cudaFree(B.queue[0]); cudaFree(B.queue[1]);
    cudaFree(B.counters); cudaFree(B.alive); cudaFree(B.tile_counts);
    cudaFree(slot_req); cudaFree(slot_g); cudaFree(counts);
    cudaFree(d_reqs); cudaFree(d_chunks); cudaFree(d_scenes);
    for (int i = 0; i < kRing; ++i) {
      cudaFreeHost(h_reqs[i]);
      cudaFreeHost(h_chunks[i]);
      if (ring_ev[i]) cudaEventDestroy(ring_ev[i]);
      if (end_ev[i]) cudaEventDestroy(end_ev[i]);
      if (prof_start[i]) cudaEventDestroy(prof_start[i]);
      if (prof_end[i]) cudaEventDestroy(prof_end[i]);
    }
    if (stream) cudaStreamDestroy(stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (pool) cudaMemPoolDestroy(pool);
  }

  bool admit(HostReq& r) {
    if (r.query) return admit_query(r);
    const size_t need = r.bytes + r.materials.size() * sizeof(float);
    if ((int)active.size() >= max_active || used + need > budget) return false;
    // stream-ordered allocation: no device-wide synchronisation while
    // other steps are in flight
    if (cudaMallocFromPoolAsync(&r.d_out, r.bytes, pool, stream) != cudaSuccess) return false;
    if (cudaMallocFromPoolAsync(&r.d_mat, r.materials.size() * sizeof(float), pool, stream) !=
        cudaSuccess) {
      cudaFreeAsync(r.d_out, stream);
      r.d_out = nullptr;
      return false;
    }
    cudaMemcpyAsync(r.d_mat, r.materials.data(), r.materials.size() * sizeof(float),
                    cudaMemcpyHostToDevice, stream);
    cudaEventCreateWithFlags(&r.done_ev, cudaEventDisableTiming);
    r.dev.P.materials = r.d_mat;
    r.dev.out = r.d_out;
    used += need;
    r.admitted = true;
    r.t_admit = now_s();
    active.push_back(r.id);
    return true;
  }

  // A ray query holds its rays (28 B each) and results (8 B each) on the
  // device from admission to release.
  bool admit_query(HostReq& r) {
    const size_t need = r.bytes;
    if ((int)active.size() >= max_active || used + need > budget) return false;
    const size_t n = (size_t)r.n_rays;
    if (cudaMallocFromPoolAsync(&r.d_rays, 28 * n, pool, stream) != cudaSuccess) return false;
    if (cudaMallocFromPoolAsync(&r.d_res, 8 * n, pool, stream) != cudaSuccess) {
      cudaFreeAsync(r.d_rays, stream);
      r.d_rays = nullptr;
      return false;
    }
    cudaMemcpyAsync(r.d_rays, r.rays.data(), 28 * n, cudaMemcpyHostToDevice, stream);
    cudaEventCreateWithFlags(&r.done_ev, cudaEventDisableTiming);
    used += need;
    r.admitted = true;
    r.t_admit = now_s();
    active.push_back(r.id);
    return true;
  }
};

namespace {

// PathParams of a request (camera basis and Parallelogram as in the frame path).
void request_params(const rq_serve_request& q, rq::PathParams& P) {
  std::memset(&P, 0, sizeof(P));
  rq::camera_basis(q.eye, q.lookat, q.up, q.hfov, q.vfov, P.cam);
  P.xres = q.xres;
  P.yres = q.yres;
  P.spp = q.spp;
  P.strata = (int)std::lround(std::sqrt((double)q.spp));
  P.max_depth = q.max_depth;
  P.rr_depth = q.rr_depth;
  P.seed = q.seed;
  for (int c = 0; c < 3; ++c) {
    P.light_anchor[c] = q.light_anchor[c];
    P.light_v1[c] = q.light_v1[c];
    P.light_v2[c] = q.light_v2[c];
    P.light_color[c] = q.light_color[c];
    P.background[c] = q.background[c];
    P.ambient[c] = q.ambient[c];
  }
  rq::environment_from(q.environment, P.env);  // checked on submit
  const float* v1 = q.light_v1;
  const float* v2 = q.light_v2;
  float n[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2],
                v1[0] * v2[1] - v1[1] * v2[0]};
  const float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  const float sc = 1 / l;
  for (int c = 0; c < 3; ++c) P.light_normal[c] = n[c] * sc;
  P.light_inv_area = (float)1 / l;
}

}  // namespace

extern "C" {

int rq_server_create(rq_scene* const* scenes, int n_scenes, long long path_capacity,
                     int chunk_pixels, size_t hbm_budget_bytes, rq_server** out) {
  using namespace rq;
  if (!out) return sfail(RQ_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!scenes || n_scenes <= 0 || n_scenes > kMaxServeScenes) return sfail(RQ_ERR_ARG, "1..32 scenes");
  if (path_capacity < 1024 || path_capacity > (1LL << 30)) return sfail(RQ_ERR_ARG, "bad path capacity");
  if (chunk_pixels <= 0 || (long long)chunk_pixels * 4096 > (1LL << 40))
    return sfail(RQ_ERR_ARG, "bad chunk_pixels");
  std::unique_ptr<rq_server> s(new rq_server());
  const Scene* s0 = reinterpret_cast<const Scene*>(scenes[0]);
  if (!s0) return sfail(RQ_ERR_ARG, "NULL scene");
  std::vector<DevScene> ds(n_scenes);
  for (int i = 0; i < n_scenes; ++i) {
    Scene* sc = reinterpret_cast<Scene*>(scenes[i]);
    if (!sc || !sc->has_tree) return sfail(RQ_ERR_STATE, "scene without a tree");
    if (sc->instanced) return sfail(RQ_ERR_ARG, "the server takes triangle scenes");
    if (sc->device != s0->device || sc->tri_kind != s0->tri_kind)
      return sfail(RQ_ERR_ARG, "scenes must share device and triangle kind");
    ds[i] = sc->dev();
    s->depth = std::max(s->depth, ds[i].depth);
    s->scenes.push_back(sc);
  }
  s->device = s0->device;
  s->tri_kind = s0->tri_kind;
  s->num_sms = s0->num_sms;
  s->n_scenes = n_scenes;
  s->capacity = path_capacity;
  s->chunk_pixels = chunk_pixels;
  s->budget = hbm_budget_bytes;
  if (cudaSetDevice(s->device) != cudaSuccess) return sfail(RQ_ERR_CUDA, "cudaSetDevice");
  const size_t C = (size_t)path_capacity;
  PathBuffers& B = s->B;
  B.capacity = C;
  bool ok = cudaMalloc(&B.o, 12 * C) == cudaSuccess && cudaMalloc(&B.d, 12 * C) == cudaSuccess &&
            cudaMalloc(&B.imp, 12 * C) == cudaSuccess && cudaMalloc(&B.rad, 12 * C) == cudaSuccess &&
            cudaMalloc(&B.rng, 8 * C) == cudaSuccess && cudaMalloc(&B.t, 4 * C) == cudaSuccess &&
            cudaMalloc(&B.pos, 4 * C) == cudaSuccess && cudaMalloc(&B.prim, 4 * C) == cudaSuccess &&
            cudaMalloc(&B.queue[0], 4 * C) == cudaSuccess &&
            cudaMalloc(&B.queue[1], 4 * C) == cudaSuccess &&
            cudaMalloc(&B.counters, kPathCounters * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&B.alive, C) == cudaSuccess &&
            cudaMalloc(&B.tile_counts, 4 * (C / 4096 + 2)) == cudaSuccess &&
            cudaMalloc(&s->slot_req, 4 * C) == cudaSuccess &&
            cudaMalloc(&s->slot_g, 8 * C) == cudaSuccess &&
            cudaMalloc(&s->counts, 16) == cudaSuccess &&
            cudaMalloc(&s->d_reqs, sizeof(ServeReq) * s->max_active) == cudaSuccess &&
            cudaMalloc(&s->d_chunks, sizeof(ServeChunk) * s->max_chunks) == cudaSuccess &&
            cudaMalloc(&s->d_scenes, sizeof(DevScene) * n_scenes) == cudaSuccess;
  ok = ok && cudaMalloc(&s->d_qdesc, sizeof(BatchDesc) * rq_server::kMaxQueryDescs) == cudaSuccess &&
       cudaMalloc(&s->d_qcounter, sizeof(int)) == cudaSuccess;
  for (int i = 0; ok && i < rq_server::kRing; ++i)
    ok = cudaMallocHost(&s->h_qdesc[i], sizeof(BatchDesc) * rq_server::kMaxQueryDescs) ==
             cudaSuccess &&
         cudaMallocHost(&s->h_reqs[i], sizeof(ServeReq) * s->max_active) == cudaSuccess &&
         cudaMallocHost(&s->h_chunks[i], sizeof(ServeChunk) * s->max_chunks) == cudaSuccess &&
         cudaEventCreateWithFlags(&s->ring_ev[i], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&s->end_ev[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) return sfail(RQ_ERR_OOM, "server pool allocation failed");
  B.ray_counts = s->counts;
  if (cudaMemset(s->counts, 0, 16) != cudaSuccess ||
      cudaMemcpy(s->d_scenes, ds.data(), sizeof(DevScene) * n_scenes, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return sfail(RQ_ERR_CUDA, "server setup");
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    uint64_t keep = ~0ull;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
      return sfail(RQ_ERR_CUDA, "server memory pool");
    // map a first slice of the budget now, so early requests do not wait
    // for the pool to grow
    void* warm = nullptr;
    const size_t first = std::min<size_t>(hbm_budget_bytes, size_t(2) << 30);
    if (cudaMallocFromPoolAsync(&warm, first, s->pool, s->stream) == cudaSuccess)
      cudaFreeAsync(warm, s->stream);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess)
      return sfail(RQ_ERR_CUDA, "server memory pool");
  }
  s->smem = (size_t)s->depth * 128 * sizeof(int2);
  s->grid = std::max(1, serve_blocks_per_sm(s->tri_kind, s->smem) * s->num_sms);
  s->qgrid = std::max(1, batch_blocks_per_sm(s->tri_kind, 0, 128, s->smem) * s->num_sms);
  s->table.assign(s->max_active, 0);
  s->host_scenes = ds;
  for (Scene* sc : s->scenes) s->generations.push_back(sc->generation);
  *out = s.release();
  return RQ_OK;
}

int rq_server_submit(rq_server* s, const rq_serve_request* q, int* request_id) {
  if (!s || !q || !request_id) return sfail(RQ_ERR_ARG, "NULL argument");
  const int strata = (int)std::lround(std::sqrt((double)q->spp));
  if (q->scene < 0 || q->scene >= s->n_scenes) return sfail(RQ_ERR_ARG, "scene index out of range");
  if (q->xres <= 0 || q->yres <= 0) return sfail(RQ_ERR_ARG, "bad resolution");
  if (q->spp <= 0 || strata * strata != q->spp) return sfail(RQ_ERR_ARG, "spp must be a perfect square");
  if ((long long)s->chunk_pixels * q->spp > s->capacity)
    return sfail(RQ_ERR_CAPACITY, "a chunk of this request does not fit the path pool");
  if (q->max_depth < 1 || q->max_depth > rq::kMaxPathDepth) return sfail(RQ_ERR_ARG, "max_depth in [1, 16]");
  if (q->n_materials <= 0 || !q->material_rgb) return sfail(RQ_ERR_ARG, "no materials");
  if (s->scenes[q->scene]->max_face_material >= q->n_materials)
    return sfail(RQ_ERR_ARG, "face_material past n_materials");
  rq::Environment env;
  if (!rq::environment_from(q->environment, env))
    return sfail(RQ_ERR_ARG, "bad environment (kind, or a zero background up)");
  const size_t bytes = (size_t)q->xres * q->yres * 12;
  if (bytes + (size_t)q->n_materials * 12 > s->budget)
    return sfail(RQ_ERR_CAPACITY, "request larger than the server's HBM budget");
  std::unique_ptr<HostReq> r(new HostReq());
  r->id = s->next_id++;
  r->spec = *q;
  r->materials.assign(q->material_rgb, q->material_rgb + 3 * q->n_materials);
  r->spec.material_rgb = nullptr;
  request_params(*q, r->dev.P);
  r->dev.scene = q->scene;
  r->bytes = bytes;
  r->npix = q->xres * q->yres;
  r->t_submit = now_s();
  *request_id = r->id;
  s->pending.push_back(r->id);
  s->reqs[r->id] = std::move(r);
  return RQ_OK;
}

int rq_server_submit_query(rq_server* s, const rq_serve_query* q, int* request_id) {
  if (!s || !q || !request_id) return sfail(RQ_ERR_ARG, "NULL argument");
  if (q->scene < 0 || q->scene >= s->n_scenes) return sfail(RQ_ERR_ARG, "scene index out of range");
  if (q->n <= 0 || q->n > (1 << 30)) return sfail(RQ_ERR_ARG, "ray count in [1, 2^30]");
  if (!q->org || !q->dir || !q->tmax) return sfail(RQ_ERR_ARG, "NULL ray arrays");
  if (q->flags != RQ_CLOSEST && q->flags != RQ_ANYHIT) return sfail(RQ_ERR_ARG, "bad flags");
  const size_t n = (size_t)q->n;
  const size_t bytes = 36 * n;
  if (bytes > s->budget) return sfail(RQ_ERR_CAPACITY, "query larger than the server's HBM budget");
  std::unique_ptr<HostReq> r(new HostReq());
  r->id = s->next_id++;
  r->query = true;
  r->n_rays = q->n;
  r->flags = q->flags;
  r->spec.scene = q->scene;
  r->rays.resize(7 * n);
  std::memcpy(r->rays.data(), q->org, 12 * n);
  std::memcpy(r->rays.data() + 3 * n, q->dir, 12 * n);
  std::memcpy(r->rays.data() + 6 * n, q->tmax, 4 * n);
  r->bytes = bytes;
  r->t_submit = now_s();
  *request_id = r->id;
  s->pending.push_back(r->id);
  s->reqs[r->id] = std::move(r);
  return RQ_OK;
}

int rq_server_query_result(rq_server* s, int request_id, float* t, int32_t* prim,
                           double* latency_s, double* queue_s) {
  if (!s) return sfail(RQ_ERR_ARG, "NULL server");
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return sfail(RQ_ERR_ARG, "unknown request");
  HostReq& r = *it->second;
  if (!r.query) return sfail(RQ_ERR_ARG, "a render request: use rq_server_result");
  if (!r.done) return sfail(RQ_ERR_STATE, "request not finished");
  if (cudaSetDevice(s->device) != cudaSuccess) return sfail(RQ_ERR_CUDA, "cudaSetDevice");
  const size_t n = (size_t)r.n_rays;
  cudaError_t e = cudaStreamWaitEvent(s->copy_stream, r.done_ev, 0);
  if (e == cudaSuccess && t)
    e = cudaMemcpyAsync(t, r.d_res, 4 * n, cudaMemcpyDeviceToHost, s->copy_stream);
  if (e == cudaSuccess && prim)
    e = cudaMemcpyAsync(prim, r.d_res + n, 4 * n, cudaMemcpyDeviceToHost, s->copy_stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->copy_stream);
  if (e != cudaSuccess) return sfail(RQ_ERR_CUDA, "query result copy failed");
  if (latency_s) *latency_s = r.t_done - r.t_submit;
  if (queue_s) *queue_s = r.t_admit - r.t_submit;
  return RQ_OK;
}

int rq_server_step(rq_server* s, int* scheduled_paths) {
  using namespace rq;
  if (!s) return sfail(RQ_ERR_ARG, "NULL server");
  if (scheduled_paths) *scheduled_paths = 0;
  if (cudaSetDevice(s->device) != cudaSuccess) return sfail(RQ_ERR_CUDA, "cudaSetDevice");
  // scenes updated since the last step: new descriptors (ordered on the
  // server's stream before this step) and a stack for the deepest tree
  bool changed = false;
  for (size_t i = 0; i < s->scenes.size(); ++i) {
    const Scene* sc = s->scenes[i];
    if (sc->generation == s->generations[i]) continue;
    if (!sc->has_tree) return sfail(RQ_ERR_STATE, "a scene of the server has no tree");
    s->host_scenes[i] = sc->dev();
    s->generations[i] = sc->generation;
    changed = true;
  }
  if (changed) {
    int depth = 1;
    for (const DevScene& d : s->host_scenes) depth = std::max(depth, d.depth);
    if (cudaMemcpyAsync(s->d_scenes, s->host_scenes.data(),
                        sizeof(DevScene) * s->host_scenes.size(), cudaMemcpyHostToDevice,
                        s->stream) != cudaSuccess)
      return sfail(RQ_ERR_CUDA, "scene table");
    if (depth != s->depth) {
      s->depth = depth;
      s->smem = (size_t)depth * 128 * sizeof(int2);
      s->grid = std::max(1, serve_blocks_per_sm(s->tri_kind, s->smem) * s->num_sms);
      s->qgrid = std::max(1, batch_blocks_per_sm(s->tri_kind, 0, 128, s->smem) * s->num_sms);
    }
  }
  // admission in arrival order while the budget allows
  while (!s->pending.empty()) {
    HostReq& r = *s->reqs[s->pending.front()];
    if (!s->admit(r)) break;
    s->pending.pop_front();
  }
  // requests with work left, in admission order: renders and ray queries
  std::vector<int> cand, qcand;
  for (int id : s->active) {
    const HostReq& r = *s->reqs[id];
    if (r.scheduled_all) continue;
    (r.query ? qcand : cand).push_back(id);
  }
  if (cand.empty() && qcand.empty()) return RQ_OK;
  const int slot = (int)(s->steps % rq_server::kRing);
  if (s->ring_used[slot] && cudaEventSynchronize(s->ring_ev[slot]) != cudaSuccess)
    return sfail(RQ_ERR_CUDA, "staging ring wait failed");
  ServeReq* hreq = s->h_reqs[slot];
  ServeChunk* hch = s->h_chunks[slot];
  std::map<int, int> tidx;  // request id -> table index this step
  int n_chunks = 0, n_req = 0, max_depth = 1;
  long long slots = 0, pix = 0;
  // Two passes over the admitted requests in admission order: first one
  // chunk each (every request advances every step), then the rest of the
  // pool oldest first, so the oldest requests - the ones whose latency is
  // the tail - get most of each step.
  auto take = [&](HostReq& r) -> bool {
    if (r.scheduled_all || n_chunks >= s->max_chunks) return false;
    const int npx = std::min(s->chunk_pixels, r.npix - r.next_pix);
    const long long need = (long long)npx * r.spec.spp;
    if (slots + need > s->capacity) return false;
    int ti;
    auto it = tidx.find(r.id);
    if (it == tidx.end()) {
      ti = n_req++;
      tidx[r.id] = ti;
      hreq[ti] = r.dev;
    } else {
      ti = it->second;
    }
    ServeChunk& c = hch[n_chunks++];
    c.req = ti;
    c.pix0 = r.next_pix;
    c.npix = npx;
    c.slot0 = (int)slots;
    c.px0 = (int)pix;
    slots += need;
    pix += npx;
    max_depth = std::max(max_depth, r.spec.max_depth);
    r.next_pix += npx;
    if (r.next_pix >= r.npix) r.scheduled_all = true;
    return true;
  };
  for (int id : cand) take(*s->reqs[id]);
  for (int id : cand)
    while (take(*s->reqs[id])) {
    }
  // Ray-query chunks, oldest request first, up to kStepQueryRays rays per
  // step: each chunk is one descriptor of the batched traversal kernel
  // over a consecutive range of the request's rays (row stride = the
  // request's ray count).
  constexpr int kQueryChunk = 1 << 20;
  constexpr long long kStepQueryRays = 8LL << 20;
  constexpr int kQueryWarpRays = 128;
  BatchDesc* hq = s->h_qdesc[slot];
  int n_qdesc = 0, q_warp_chunks = 0;
  long long qrays = 0;
  std::vector<int> qstep;  // query requests with rays in this step
  for (int id : qcand) {
    HostReq& r = *s->reqs[id];
    bool any_here = false;
    while (r.next_ray < r.n_rays && qrays < kStepQueryRays &&
           n_qdesc < rq_server::kMaxQueryDescs) {
      const int cnt = (int)std::min<long long>(
          {(long long)kQueryChunk, (long long)(r.n_rays - r.next_ray), kStepQueryRays - qrays});
      const size_t n = (size_t)r.n_rays, r0 = (size_t)r.next_ray;
      BatchDesc& d = hq[n_qdesc++];
      d.scene = r.spec.scene;
      d.n = cnt;
      d.any = r.flags == RQ_ANYHIT;
      d.chunk0 = q_warp_chunks;
      d.org = r.d_rays + r0;
      d.dir = r.d_rays + 3 * n + r0;
      d.tmax = r.d_rays + 6 * n + r0;
      d.t = r.d_res + r0;
      d.prim = reinterpret_cast<int32_t*>(r.d_res + n) + r0;
      d.u = nullptr;
      d.v = nullptr;
      d.stride = r.n_rays;
      q_warp_chunks += (cnt + kQueryWarpRays - 1) / kQueryWarpRays;
      qrays += cnt;
      r.next_ray += cnt;
      any_here = true;
    }
    if (r.next_ray >= r.n_rays) r.scheduled_all = true;
    if (any_here) qstep.push_back(id);
  }
  if (n_chunks == 0 && n_qdesc == 0) return RQ_OK;
  cudaStream_t st = s->stream;
  cudaError_t e = cudaSuccess;
  if (n_chunks > 0) {
    e = cudaMemcpyAsync(s->d_reqs, hreq, sizeof(ServeReq) * n_req, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->d_chunks, hch, sizeof(ServeChunk) * n_chunks, cudaMemcpyHostToDevice,
                          st);
  }
  if (e == cudaSuccess && n_qdesc > 0)
    e = cudaMemcpyAsync(s->d_qdesc, hq, sizeof(BatchDesc) * n_qdesc, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaEventRecord(s->ring_ev[slot], st);
  s->ring_used[slot] = true;
  if (s->profile) {
    s->close_profile(slot, true);
    std::vector<int> seen;
    for (int i = 0; i < n_req; ++i)
      if (std::find(seen.begin(), seen.end(), hreq[i].scene) == seen.end())
        seen.push_back(hreq[i].scene);
    rq_server_step_record& pr = s->prof_slot[slot];
    pr.requests = n_req;
    pr.chunks = n_chunks;
    pr.scenes = (int)seen.size();
    pr.max_depth = max_depth;
    pr.paths = slots;
    pr.gpu_ms = 0.f;
    pr.t_enqueue_s = now_s() - s->prof_t0;
    s->prof_open[slot] = true;
    if (e == cudaSuccess) e = cudaEventRecord(s->prof_start[slot], st);
  }
  // the step's ray queries: one persistent launch of the batched kernel
  if (e == cudaSuccess && n_qdesc > 0) {
    BatchArgs Q{};
    Q.scenes = s->d_scenes;
    Q.n_scenes = s->n_scenes;
    Q.batches = s->d_qdesc;
    Q.n_batches = n_qdesc;
    Q.total_chunks = q_warp_chunks;
    Q.chunk_rays = kQueryWarpRays;
    Q.refill = 8;
    Q.stack_depth = s->depth;
    Q.counter = s->d_qcounter;
    Q.stats = nullptr;
    e = cudaMemsetAsync(s->d_qcounter, 0, sizeof(int), st);
    const int qg = std::max(1, std::min(s->qgrid, (q_warp_chunks * 32 + 127) / 128));
    if (e == cudaSuccess) e = launch_batch(s->tri_kind, 0, Q, qg, 128, s->smem, st);
    s->query_rays += (unsigned long long)qrays;
  }
  // the step's path chunks: one wavefront over all of them
  if (e == cudaSuccess && n_chunks > 0) {
    ServeArgs A;
    A.scenes = s->d_scenes;
    A.n_scenes = s->n_scenes;
    A.reqs = s->d_reqs;
    A.chunks = s->d_chunks;
    A.n_chunks = n_chunks;
    A.n_slots = (int)slots;
    A.n_pix = (int)pix;
    A.slot_req = s->slot_req;
    A.slot_g = s->slot_g;
    e = s->tri_kind == kWald ? serve_launch_step<kWald>(A, s->B, max_depth, s->grid, s->smem, st)
                             : serve_launch_step<kKS>(A, s->B, max_depth, s->grid, s->smem, st);
  }
  if (e != cudaSuccess) return sfail(RQ_ERR_CUDA, std::string("serve step: ") + cudaGetErrorString(e));
  for (auto& kv : tidx) {
    HostReq& r = *s->reqs[kv.first];
    if (r.scheduled_all) cudaEventRecord(r.done_ev, st);
  }
  for (int id : qstep) {
    HostReq& r = *s->reqs[id];
    if (r.scheduled_all) cudaEventRecord(r.done_ev, st);
  }
  cudaEventRecord(s->end_ev[slot], st);
  if (s->profile) cudaEventRecord(s->prof_end[slot], st);
  ++s->steps;
  if (scheduled_paths) *scheduled_paths = (int)std::min<long long>(slots + qrays, 1LL << 30);
  // keep at most two steps in flight: wait for the end of the step before
  // the one just enqueued
  if (s->steps >= 2) {
    const int prev = (int)((s->steps - 2) % rq_server::kRing);
    if (cudaEventSynchronize(s->end_ev[prev]) != cudaSuccess)
      return sfail(RQ_ERR_CUDA, "serve step failed on the device");
  }
  return RQ_OK;
}

int rq_server_poll(rq_server* s, int* done_ids, int max_ids, int* n_done) {
  if (!s || !n_done) return sfail(RQ_ERR_ARG, "NULL argument");
  *n_done = 0;
  const double t = now_s();
  std::vector<int> still;
  for (int id : s->active) {
    HostReq& r = *s->reqs[id];
    if (r.scheduled_all && !r.done && cudaEventQuery(r.done_ev) == cudaSuccess) {
      r.done = true;
      r.t_done = t;
    }
    if (r.done) {
      if (*n_done < max_ids && done_ids) done_ids[(*n_done)++] = id;
      else if (!done_ids) ++*n_done;
    } else {
      still.push_back(id);
    }
  }
  s->active.swap(still);
  return RQ_OK;
}

int rq_server_result(rq_server* s, int request_id, float* rgb, double* latency_s,
                     double* queue_s) {
  if (!s) return sfail(RQ_ERR_ARG, "NULL server");
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return sfail(RQ_ERR_ARG, "unknown request");
  HostReq& r = *it->second;
  if (r.query) return sfail(RQ_ERR_ARG, "a ray-query request: use rq_server_query_result");
  if (!r.done) return sfail(RQ_ERR_STATE, "request not finished");
  if (cudaSetDevice(s->device) != cudaSuccess) return sfail(RQ_ERR_CUDA, "cudaSetDevice");
  if (rgb && (cudaStreamWaitEvent(s->copy_stream, r.done_ev, 0) != cudaSuccess ||
              cudaMemcpyAsync(rgb, r.d_out, r.bytes, cudaMemcpyDeviceToHost, s->copy_stream) !=
                  cudaSuccess ||
              cudaStreamSynchronize(s->copy_stream) != cudaSuccess))
    return sfail(RQ_ERR_CUDA, "result copy failed");
  if (latency_s) *latency_s = r.t_done - r.t_submit;
  if (queue_s) *queue_s = r.t_admit - r.t_submit;
  return RQ_OK;
}

int rq_server_release(rq_server* s, int request_id) {
  if (!s) return sfail(RQ_ERR_ARG, "NULL server");
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return sfail(RQ_ERR_ARG, "unknown request");
  HostReq& r = *it->second;
  if (r.admitted && !r.done) return sfail(RQ_ERR_STATE, "request still running");
  cudaSetDevice(s->device);
  if (r.admitted) s->used -= r.bytes + r.materials.size() * sizeof(float);
  if (r.d_out) cudaFreeAsync(r.d_out, s->stream);
  if (r.d_mat) cudaFreeAsync(r.d_mat, s->stream);
  if (r.d_rays) cudaFreeAsync(r.d_rays, s->stream);
  if (r.d_res) cudaFreeAsync(r.d_res, s->stream);
  if (r.done_ev) cudaEventDestroy(r.done_ev);
  if (!r.admitted) {
    for (auto p = s->pending.begin(); p != s->pending.end(); ++p)
      if (*p == request_id) {
        s->pending.erase(p);
        break;
      }
  }
  s->reqs.erase(it);
  return RQ_OK;
}

int rq_server_stats(rq_server* s, uint64_t* ray_counts, long long* steps, int* pending,
                     int* active, size_t* bytes_in_use) {
  if (!s) return sfail(RQ_ERR_ARG, "NULL server");
  cudaSetDevice(s->device);
  if (ray_counts) {
    cudaStreamSynchronize(s->stream);
    if (cudaMemcpy(ray_counts, s->counts, 16, cudaMemcpyDeviceToHost) != cudaSuccess)
      return sfail(RQ_ERR_CUDA, "counter copy failed");
    ray_counts[0] += s->query_rays;  // ray-query rays count as traced rays
  }
  if (steps) *steps = s->steps;
  if (pending) *pending = (int)s->pending.size();
  if (active) *active = (int)s->active.size();
  if (bytes_in_use) *bytes_in_use = s->used;
  return RQ_OK;
}

int rq_server_destroy(rq_server* s) {
  delete s;
  return RQ_OK;
}

int rq_server_set_profile(rq_server* s, int on) {
  if (!s) return sfail(RQ_ERR_ARG, "NULL server");
  if (cudaSetDevice(s->device) != cudaSuccess) return sfail(RQ_ERR_CUDA, "cudaSetDevice");
  if (on && !s->prof_start[0]) {
    for (int i = 0; i < rq_server::kRing; ++i)
      if (cudaEventCreate(&s->prof_start[i]) != cudaSuccess ||
          cudaEventCreate(&s->prof_end[i]) != cudaSuccess)
        return sfail(RQ_ERR_CUDA, "profile events");
  }
  if (!on)
    for (int i = 0; i < rq_server::kRing; ++i) s->close_profile(i, true);
  s->profile = on != 0;
  s->prof_t0 = now_s();
  return RQ_OK;
}

int rq_server_profile(rq_server* s, rq_server_step_record* out, int max_steps, int* n_steps) {
  if (!s || !n_steps || (max_steps > 0 && !out)) return sfail(RQ_ERR_ARG, "NULL argument");
  if (cudaSetDevice(s->device) != cudaSuccess) return sfail(RQ_ERR_CUDA, "cudaSetDevice");
  for (int i = 0; i < rq_server::kRing; ++i) s->close_profile(i, false);
  const int n = std::min<int>(max_steps, (int)s->prof_done.size());
  std::copy(s->prof_done.begin(), s->prof_done.begin() + n, out);
  s->prof_done.erase(s->prof_done.begin(), s->prof_done.begin() + n);
  *n_steps = n;
  return RQ_OK;
}

int rq_server_run_stream(rq_server* s, const rq_serve_request* requests,
                         const double* arrival_s, int n, float* const* images,
                         double* latency_s, double* queue_s, double* wall_s, double timeout_s) {
  if (!s || (n > 0 && (!requests || !arrival_s || !latency_s))) return sfail(RQ_ERR_ARG, "NULL argument");
  if (n < 0) return sfail(RQ_ERR_ARG, "negative request count");
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return arrival_s[a] < arrival_s[b]; });
  std::map<int, int> index_of;  // request id -> position in `requests`
  std::vector<int> done_ids(1024);
  const double t0 = now_s();
  double first = -1, last = t0;
  int k = 0, done = 0;
  while (done < n) {
    const double now = now_s() - t0;
    if (now > timeout_s) return sfail(RQ_ERR_TIMEOUT, "serving stream did not finish in time");
    while (k < n && arrival_s[order[k]] <= now) {
      int id = 0;
      const int rc = rq_server_submit(s, &requests[order[k]], &id);
      if (rc != RQ_OK) return rc;
      if (first < 0) first = now_s();
      index_of[id] = order[k++];
    }
    int scheduled = 0;
    int rc = rq_server_step(s, &scheduled);
    if (rc != RQ_OK) return rc;
    int nd = 0;
    rc = rq_server_poll(s, done_ids.data(), (int)done_ids.size(), &nd);
    if (rc != RQ_OK) return rc;
    for (int j = 0; j < nd; ++j) {
      const int i = index_of[done_ids[j]];
      double lat = 0, qs = 0;
      rc = rq_server_result(s, done_ids[j], images ? images[i] : nullptr, &lat, &qs);
      if (rc != RQ_OK) return rc;
      latency_s[i] = lat;
      if (queue_s) queue_s[i] = qs;
      rc = rq_server_release(s, done_ids[j]);
      if (rc != RQ_OK) return rc;
      last = now_s();
      ++done;
    }
    if (scheduled == 0 && nd == 0) {
      // nothing new to enqueue: sleep until the next arrival or a short
      // interval (steps in flight finish meanwhile)
      double wait = 2e-5;
      if (k < n && s->active.empty()) wait = std::max(0.0, arrival_s[order[k]] - (now_s() - t0));
      std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 5e-4)));
    }
  }
  if (wall_s) *wall_s = n > 0 ? last - first : 0.0;
  return RQ_OK;
}

}  // extern "C"
