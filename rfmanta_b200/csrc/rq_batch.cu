// Batched ray queries: many batches of uneven size, closest hit or any hit,
// over several resident scenes, in ONE persistent launch.
//
// Work is cut into chunks of `chunk_rays` consecutive rays of one batch.
// Each warp claims a chunk with one atomicAdd and hands its rays to idle
// lanes; after every while-while step the warp counts idle lanes with a
// ballot and refills them (from the current chunk, claiming the next chunk
// when it runs dry) once `refill` or more are idle or none is busy.  A warp
// can therefore hold rays of different batches, scenes and query kinds at
// the same time; each lane keeps its own batch, scene and any-hit flag.
// Scene descriptors are staged in shared memory; the traversal stack keeps
// `R` entries in registers and spills to the thread's shared-memory column
// (sized to the deepest scene).
//
// A plan uploads the scene and batch tables once and captures the launch
// (counter reset + kernel) in a CUDA graph; rq_batch_plan_launch replays it.
// rq_batch_autotune times candidate configurations on the real batches and
// returns the fastest.  Results do not depend on the configuration: every
// ray is traced by the same per-ray procedure (tested).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_batch.h"
#include "rq_scene.h"
#include "rq_traverse.cuh"

namespace rq {

// Resets a lane's traversal stack: a RegStack over the thread's shared
// column, or a SplitStack whose first A.stack_depth entries sit there and
// whose deeper ones go to the thread's entries of the overflow area.
template <int R>
__device__ __forceinline__ void reset_stack(RegStack<R>& st, int2* smem, const BatchArgs&) {
  st.init(smem + threadIdx.x, blockDim.x);
}
__device__ __forceinline__ void reset_stack(SplitStack& st, int2* smem, const BatchArgs& A) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  st.init(smem + threadIdx.x, A.stack_depth, A.ovf + g);
}

// SPLIT: the stack is a SplitStack with a short shared column, and
// registers are held to 48 per thread (five 256-thread blocks per SM), so
// more warps are resident to hide the traversal's dependent loads.
template <int KIND, int R, bool STATS, bool SPLIT>
__global__ void __launch_bounds__(256, SPLIT ? 5 : 1) batch_kernel(BatchArgs A) {
  extern __shared__ int2 smem[];
  __shared__ DevScene sm_scenes[kMaxBatchScenes];
  for (int i = threadIdx.x; i < A.n_scenes; i += blockDim.x) sm_scenes[i] = A.scenes[i];
  __syncthreads();
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  typename std::conditional<SPLIT, SplitStack, RegStack<R>>::type st;
  reset_stack(st, smem, A);
  // warp-uniform chunk state
  int w_batch = 0, w_next = 0, w_end = 0;
  bool exhausted = false;
  // lane state
  int my_ray = -1;
  int my_tag = 0;  // batch << 6 | scene << 1 | any hit (one register for the three)
  Ray r;
  Hit h;
  int ref = kDone;
  Counts cnt;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, my_ray < 0);
    const unsigned busy = ~idle;
    if (!exhausted && idle && (__popc(idle) >= A.refill || busy == 0u)) {
      unsigned need = idle;
      while (need) {
        if (w_next >= w_end) {
          int c = 0;
          if (lane == 0) c = atomicAdd(A.counter, 1);
          c = __shfl_sync(0xffffffffu, c, 0);
          if (c >= A.total_chunks) {
            exhausted = true;
            break;
          }
          int lo = 0, hi = A.n_batches - 1;  // last batch with chunk0 <= c
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(&A.batches[mid].chunk0) <= c) lo = mid;
            else hi = mid - 1;
          }
          w_batch = lo;
          w_next = (c - __ldg(&A.batches[lo].chunk0)) * A.chunk_rays;
          w_end = min(w_next + A.chunk_rays, __ldg(&A.batches[lo].n));
        }
        const int k = min(__popc(need), w_end - w_next);
        const bool take = ((need >> lane) & 1u) && (int)__popc(need & lt) < k;
        if (take) {
          const BatchDesc& B = A.batches[w_batch];
          my_ray = w_next + (int)__popc(need & lt);
          my_tag = (w_batch << 6) | (B.scene << 1) | (B.any != 0);
          const int n = B.stride ? B.stride : B.n;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            r.o[c] = __ldg(B.org + (size_t)c * n + my_ray);
            r.d[c] = __ldg(B.dir + (size_t)c * n + my_ray);
            r.inv[c] = fdiv(1.f, r.d[c]);
          }
          r.minT = __ldg(B.tmax + my_ray);
          int sp0;
          start_ray(sm_scenes[B.scene], r, h, ref, sp0);
          reset_stack(st, smem, A);
          if (STATS) cnt.boxes += 1;
        }
        const unsigned taken = __ballot_sync(0xffffffffu, take);
        need &= ~taken;
        w_next += k;
      }
    }
    if (exhausted && __all_sync(0xffffffffu, my_ray < 0)) break;
    // Work is ordered scene by scene, closest-hit batches before any-hit
    // ones, so a warp's busy lanes almost always share the query kind: the
    // step is then compiled for that kind (the per-lane form only where
    // kinds meet).
    const bool stepping = my_ray >= 0 && ref != kDone;
    const bool my_any = (my_tag & 1) != 0;
    const int my_scene = (my_tag >> 1) & 31;
    const unsigned any_m = __ballot_sync(0xffffffffu, stepping && my_any);
    const unsigned clo_m = __ballot_sync(0xffffffffu, stepping && !my_any);
    if (my_ray >= 0) {
      if (stepping) {
        // the lane's scene descriptor copied to registers: the step's stack
        // stores go to shared memory too, and a descriptor read from there
        // would be read again after every store
        DevScene S;
        S.nodes = sm_scenes[my_scene].nodes;
        S.tris = sm_scenes[my_scene].tris;
        if (any_m == 0u)
          step_dyn<KIND, R, STATS>(S, r, h, ref, st, false, &cnt);
        else if (clo_m == 0u)
          step_dyn<KIND, R, STATS>(S, r, h, ref, st, true, &cnt);
        else
          step_dyn<KIND, R, STATS>(S, r, h, ref, st, my_any, &cnt);
      }
      if (ref == kDone) {
        const BatchDesc& B = A.batches[my_tag >> 6];
        if (B.t) B.t[my_ray] = h.t;
        if (B.prim) B.prim[my_ray] = h.id;
        if (B.u) B.u[my_ray] = h.u;
        if (B.v) B.v[my_ray] = h.v;
        my_ray = -1;
      }
    }
  }
  if (STATS) {
    atomicAdd(&A.stats[0], (unsigned long long)cnt.boxes);
    atomicAdd(&A.stats[1], (unsigned long long)cnt.tris);
  }
}

template <int KIND, int R, bool STATS, bool SPLIT = false>
static cudaError_t batch_go(bool launch, int grid, int block, size_t smem, const BatchArgs& A,
                            cudaStream_t st, const void** fn) {
  if (fn) *fn = (const void*)batch_kernel<KIND, R, STATS, SPLIT>;
  if (launch) batch_kernel<KIND, R, STATS, SPLIT><<<grid, block, smem, st>>>(A);
  return launch ? cudaGetLastError() : cudaSuccess;
}

// Resolves (triangle kind, register stack, statistics) to one kernel and
// either returns its address or launches it; reg = kSplitStack selects the
// split-stack kernel.
constexpr int kSplitStack = -1;
template <int KIND>
static cudaError_t batch_dispatch_kind(int reg, bool stats, bool launch, int grid, int block,
                                       size_t smem, const BatchArgs& A, cudaStream_t st,
                                       const void** fn) {
  switch (reg) {
    case kSplitStack:
      return stats ? batch_go<KIND, 0, true, true>(launch, grid, block, smem, A, st, fn)
                   : batch_go<KIND, 0, false, true>(launch, grid, block, smem, A, st, fn);
    case 1:
      return stats ? batch_go<KIND, 1, true>(launch, grid, block, smem, A, st, fn)
                   : batch_go<KIND, 1, false>(launch, grid, block, smem, A, st, fn);
    case 2:
      return stats ? batch_go<KIND, 2, true>(launch, grid, block, smem, A, st, fn)
                   : batch_go<KIND, 2, false>(launch, grid, block, smem, A, st, fn);
    case 4:
      return stats ? batch_go<KIND, 4, true>(launch, grid, block, smem, A, st, fn)
                   : batch_go<KIND, 4, false>(launch, grid, block, smem, A, st, fn);
    default:
      return stats ? batch_go<KIND, 0, true>(launch, grid, block, smem, A, st, fn)
                   : batch_go<KIND, 0, false>(launch, grid, block, smem, A, st, fn);
  }
}

static cudaError_t batch_dispatch(int kind, int reg, bool stats, bool launch, int grid,
                                  int block, size_t smem, const BatchArgs& A, cudaStream_t st,
                                  const void** fn) {
  if (kind == kWald)
    return batch_dispatch_kind<kWald>(reg, stats, launch, grid, block, smem, A, st, fn);
  return batch_dispatch_kind<kKS>(reg, stats, launch, grid, block, smem, A, st, fn);
}

cudaError_t launch_batch(int tri_kind, int reg_stack, const BatchArgs& A, int grid, int block,
                         size_t smem, cudaStream_t st) {
  const void* f = nullptr;
  batch_dispatch(tri_kind, reg_stack, A.stats != nullptr, false, 0, 0, 0, A, nullptr, &f);
  // static shared memory (the scene table) counts against the default 48 KB
  // too, so the dynamic size is always declared
  if (smem > 0)
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return batch_dispatch(tri_kind, reg_stack, A.stats != nullptr, true, grid, block, smem, A, st,
                        nullptr);
}

int batch_blocks_per_sm(int tri_kind, int reg_stack, int block, size_t smem) {
  const void* f = nullptr;
  BatchArgs A{};
  batch_dispatch(tri_kind, reg_stack, false, false, 0, 0, 0, A, nullptr, &f);
  if (smem > 0)
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, block, smem) != cudaSuccess) b = 1;
  return std::max(1, b);
}

}  // namespace rq

struct rq_batch_plan {
  int device = 0;
  int tri_kind = 0;
  rq_batch_config cfg{};
  rq::BatchArgs args{};
  rq::DevScene* d_scenes = nullptr;
  rq::BatchDesc* d_batches = nullptr;
  int* d_counter = nullptr;
  int2* d_ovf = nullptr;  // split-stack overflow area
  size_t ovf_bytes = 0;
  int grid = 1;
  size_t smem = 0;
  long long total_rays = 0;
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // the scenes' descriptors as captured, and their generations: a scene
  // updated since (refit, rotations, new tree) gets its descriptor copied
  // in again before the next launch
  std::vector<rq::Scene*> scenes;
  std::vector<uint64_t> generations;
  std::vector<rq::DevScene> host_scenes;
  int stack_depth = 1;
  int num_sms = 148;
  ~rq_batch_plan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    cudaFree(d_scenes);
    cudaFree(d_batches);
    cudaFree(d_counter);
    cudaFree(d_ovf);
  }
};

namespace {

int bfail(int code, const std::string& m) {
  rq::set_error(m);
  return code;
}

rq_batch_config default_batch_config() {
  rq_batch_config c;
  c.block_threads = 128;
  c.blocks_per_sm = 0;
  c.chunk_rays = 128;
  c.refill_threshold = 8;
  c.reg_stack = 0;
  c.node_layout = RQ_LAYOUT_DFS;
  c.smem_entries = 0;
  return c;
}

// Sizes the traversal stack for the plan's deepest tree and captures
// counter reset + persistent launch in a graph (again after a scene's tree
// grew deeper).
int capture_plan(rq_batch_plan* p) {
  using namespace rq;
  const rq_batch_config& cfg = p->cfg;
  BatchArgs& A = p->args;
  // split stack: the first smem_entries entries in shared memory, the rest
  // of the deepest tree's entries in the overflow area
  const bool split = cfg.smem_entries > 0;
  const int reg = split ? kSplitStack : cfg.reg_stack;
  A.stack_depth = split ? std::min(cfg.smem_entries, p->stack_depth) : p->stack_depth;
  // the shared-memory column holds what the register entries do not
  p->smem = (size_t)std::max(1, A.stack_depth - (split ? 0 : cfg.reg_stack)) *
            cfg.block_threads * sizeof(int2);
  const bool stats = A.stats != nullptr;
  const void* f = nullptr;
  batch_dispatch(p->tri_kind, reg, stats, false, 0, 0, 0, A, nullptr, &f);
  if (p->smem > 0 &&
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem) !=
          cudaSuccess)
    return bfail(RQ_ERR_CAPACITY, "traversal stack does not fit in shared memory");
  int bps = cfg.blocks_per_sm;
  if (bps <= 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, f, cfg.block_threads, p->smem) !=
            cudaSuccess ||
        bps <= 0)
      bps = 1;
  }
  const long long warps_needed = A.total_chunks;  // at most one chunk per warp to start
  const long long max_blocks =
      std::max(1LL, (warps_needed * 32 + cfg.block_threads - 1) / cfg.block_threads);
  p->grid = (int)std::max(1LL, std::min((long long)bps * p->num_sms, max_blocks));
  if (split) {
    const size_t need =
        (size_t)(p->stack_depth - A.stack_depth) * p->grid * cfg.block_threads * sizeof(int2);
    if (need > p->ovf_bytes) {
      // launches of the graph captured before may still use the old area
      cudaDeviceSynchronize();
      cudaFree(p->d_ovf);
      p->d_ovf = nullptr;
      p->ovf_bytes = 0;
      if (cudaMalloc(&p->d_ovf, need) != cudaSuccess)
        return bfail(RQ_ERR_OOM, "traversal stack overflow area");
      p->ovf_bytes = need;
    }
    A.ovf = p->d_ovf;
  }
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->exec = nullptr;
  p->graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaMemsetAsync(p->d_counter, 0, sizeof(int), p->cap_stream);
    batch_dispatch(p->tri_kind, reg, stats, true, p->grid, cfg.block_threads, p->smem, A,
                   p->cap_stream, nullptr);
    e = cudaStreamEndCapture(p->cap_stream, &p->graph);
  }
  if (e == cudaSuccess && split) {
    // split stack: the shared-memory carveout is set to what the resident
    // blocks use (column + scene table + the per-block reservation), so the
    // rest of the SM's L1/shared storage caches node and triangle records
    int dev = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, f);
    const size_t need = (size_t)bps * (p->smem + fa.sharedSizeBytes + 1024);
    if (per_sm > 0) {
      cudaLaunchAttributeValue v{};
      v.sharedMemCarveout =
          (unsigned)std::min<size_t>(100, (need * 100 + per_sm - 1) / per_sm);
      size_t n = 0;
      cudaGraphGetNodes(p->graph, nullptr, &n);
      std::vector<cudaGraphNode_t> nodes(n);
      cudaGraphGetNodes(p->graph, nodes.data(), &n);
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
          e = cudaGraphKernelNodeSetAttribute(nd, cudaLaunchAttributePreferredSharedMemoryCarveout,
                                              &v);
      }
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
  if (e != cudaSuccess) return bfail(RQ_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
  return RQ_OK;
}

}  // namespace

extern "C" {

int rq_batch_plan_create(rq_scene* const* scenes, int n_scenes, const rq_batch* batches,
                         int n_batches, const rq_batch_config* cfg_in, rq_batch_plan** out) {
  using namespace rq;
  if (!out) return bfail(RQ_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!scenes || n_scenes <= 0 || n_scenes > kMaxBatchScenes)
    return bfail(RQ_ERR_ARG, "1..32 scenes");
  if (!batches || n_batches <= 0) return bfail(RQ_ERR_ARG, "no batches");
  if (n_batches > (1 << 24)) return bfail(RQ_ERR_CAPACITY, "more than 2^24 batches");
  rq_batch_config cfg = cfg_in ? *cfg_in : default_batch_config();
  if (cfg.block_threads < 32 || cfg.block_threads > 256 || cfg.block_threads % 32)
    return bfail(RQ_ERR_ARG, "block_threads must be a multiple of 32 in [32, 256]");
  if (cfg.chunk_rays < 32 || cfg.chunk_rays % 32 || cfg.chunk_rays > (1 << 20))
    return bfail(RQ_ERR_ARG, "chunk_rays must be a multiple of 32");
  if (cfg.refill_threshold < 1 || cfg.refill_threshold > 32)
    return bfail(RQ_ERR_ARG, "refill_threshold must be in [1, 32]");
  if (cfg.reg_stack != 0 && cfg.reg_stack != 1 && cfg.reg_stack != 2 && cfg.reg_stack != 4)
    return bfail(RQ_ERR_ARG, "reg_stack is 0, 1, 2 or 4");
  if (cfg.node_layout < RQ_LAYOUT_DFS || cfg.node_layout > RQ_LAYOUT_BFS_TOP)
    return bfail(RQ_ERR_ARG, "node_layout is one of RQ_LAYOUT_*");
  if (cfg.smem_entries < 0 || cfg.smem_entries > 64)
    return bfail(RQ_ERR_ARG, "smem_entries must be in [0, 64]");
  if (cfg.smem_entries > 0 && cfg.reg_stack != 0)
    return bfail(RQ_ERR_ARG, "smem_entries > 0 takes reg_stack 0");
  const Scene* s0 = reinterpret_cast<const Scene*>(scenes[0]);
  if (!s0) return bfail(RQ_ERR_ARG, "NULL scene");
  if (cudaSetDevice(s0->device) != cudaSuccess) return bfail(RQ_ERR_CUDA, "cudaSetDevice");
  std::vector<DevScene> ds(n_scenes);
  int depth = 1;
  for (int i = 0; i < n_scenes; ++i) {
    Scene* s = reinterpret_cast<Scene*>(scenes[i]);
    if (!s) return bfail(RQ_ERR_ARG, "NULL scene");
    if (!s->has_tree) return bfail(RQ_ERR_STATE, "scene " + std::to_string(i) + " has no tree");
    if (s->instanced) return bfail(RQ_ERR_ARG, "batched queries take triangle scenes");
    if (s->device != s0->device) return bfail(RQ_ERR_ARG, "all scenes must be on one device");
    if (s->tri_kind != s0->tri_kind) return bfail(RQ_ERR_ARG, "all scenes must use one triangle kind");
    const int rc = s->node_layout(cfg.node_layout, ds[i]);
    if (rc != RQ_OK) return rc;
    depth = std::max(depth, ds[i].depth);
  }
  // Work order: scene by scene (closest-hit batches, then any-hit, each in
  // submission order), so the warps resident at any moment mostly trace
  // one scene and share its node and triangle records in L1/L2, as a
  // plain per-batch launch does, instead of all scenes at once.
  std::vector<int> order(n_batches);
  for (int b = 0; b < n_batches; ++b) order[b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    if (batches[a].scene != batches[b].scene) return batches[a].scene < batches[b].scene;
    return batches[a].flags < batches[b].flags;
  });
  std::vector<BatchDesc> bd(n_batches);
  int chunks = 0;
  long long rays = 0;
  for (int k = 0; k < n_batches; ++k) {
    const int b = k;
    const rq_batch& q = batches[order[k]];
    if (q.scene < 0 || q.scene >= n_scenes) return bfail(RQ_ERR_ARG, "batch scene index out of range");
    if (q.n < 0 || (q.n > 0 && (!q.d_org || !q.d_dir || !q.d_tmax)))
      return bfail(RQ_ERR_ARG, "bad batch ray arrays");
    if (q.flags != RQ_CLOSEST && q.flags != RQ_ANYHIT) return bfail(RQ_ERR_ARG, "bad batch flags");
    BatchDesc& d = bd[b];
    d.scene = q.scene;
    d.n = q.n;
    d.any = q.flags == RQ_ANYHIT;
    d.chunk0 = chunks;
    d.org = q.d_org;
    d.dir = q.d_dir;
    d.tmax = q.d_tmax;
    d.t = q.d_t;
    d.prim = q.d_prim;
    d.u = q.d_u;
    d.v = q.d_v;
    d.stride = 0;
    const long long c = ((long long)q.n + cfg.chunk_rays - 1) / cfg.chunk_rays;
    if (chunks + c > (1LL << 30)) return bfail(RQ_ERR_CAPACITY, "too many chunks");
    chunks += (int)c;
    rays += q.n;
  }
  if (cudaSetDevice(s0->device) != cudaSuccess) return bfail(RQ_ERR_CUDA, "cudaSetDevice");
  std::unique_ptr<rq_batch_plan> p(new rq_batch_plan());
  p->device = s0->device;
  p->tri_kind = s0->tri_kind;
  p->cfg = cfg;
  p->total_rays = rays;
  if (cudaMalloc(&p->d_scenes, sizeof(DevScene) * n_scenes) != cudaSuccess ||
      cudaMalloc(&p->d_batches, sizeof(BatchDesc) * n_batches) != cudaSuccess ||
      cudaMalloc(&p->d_counter, sizeof(int)) != cudaSuccess)
    return bfail(RQ_ERR_OOM, "plan tables");
  if (cudaMemcpy(p->d_scenes, ds.data(), sizeof(DevScene) * n_scenes, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(p->d_batches, bd.data(), sizeof(BatchDesc) * n_batches,
                 cudaMemcpyHostToDevice) != cudaSuccess)
    return bfail(RQ_ERR_CUDA, "plan table upload");
  BatchArgs& A = p->args;
  A.scenes = p->d_scenes;
  A.n_scenes = n_scenes;
  A.batches = p->d_batches;
  A.n_batches = n_batches;
  A.total_chunks = chunks;
  A.chunk_rays = cfg.chunk_rays;
  A.refill = cfg.refill_threshold;
  A.counter = p->d_counter;
  A.stats = s0->stats;
  p->num_sms = s0->num_sms;
  p->stack_depth = depth;
  p->host_scenes = ds;
  for (int i = 0; i < n_scenes; ++i) {
    Scene* s = reinterpret_cast<Scene*>(scenes[i]);
    p->scenes.push_back(s);
    p->generations.push_back(s->generation);
  }
  if (cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
    return bfail(RQ_ERR_CUDA, "stream");
  const int rc = capture_plan(p.get());
  if (rc != RQ_OK) return rc;
  *out = p.release();
  return RQ_OK;
}

int rq_batch_plan_launch(rq_batch_plan* plan, void* stream) {
  if (!plan) return bfail(RQ_ERR_ARG, "NULL plan");
  if (cudaSetDevice(plan->device) != cudaSuccess) return bfail(RQ_ERR_CUDA, "cudaSetDevice");
  bool changed = false;
  for (size_t i = 0; i < plan->scenes.size(); ++i) {
    rq::Scene* s = plan->scenes[i];
    if (s->generation == plan->generations[i]) continue;
    if (!s->has_tree) return bfail(RQ_ERR_STATE, "a scene of the plan has no tree");
    // the plan's node layout of the new tree (made again on the device)
    const int rc = s->node_layout(plan->cfg.node_layout, plan->host_scenes[i]);
    if (rc != RQ_OK) return rc;
    plan->generations[i] = s->generation;
    changed = true;
  }
  if (changed) {
    int depth = 1;
    for (const rq::DevScene& d : plan->host_scenes) depth = std::max(depth, d.depth);
    if (depth > plan->stack_depth) {
      // a deeper tree: a larger stack, captured again (after the launches
      // already queued, which still use the old graph)
      plan->stack_depth = depth;
      const int rc = capture_plan(plan);
      if (rc != RQ_OK) return rc;
    }
    // ordered before this launch on its stream (pageable source: the copy
    // is staged before the call returns)
    const cudaError_t c =
        cudaMemcpyAsync(plan->d_scenes, plan->host_scenes.data(),
                        sizeof(rq::DevScene) * plan->host_scenes.size(), cudaMemcpyHostToDevice,
                        static_cast<cudaStream_t>(stream));
    if (c != cudaSuccess) return bfail(RQ_ERR_CUDA, "scene table");
  }
  const cudaError_t e = cudaGraphLaunch(plan->exec, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return bfail(RQ_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
  return RQ_OK;
}

int rq_batch_plan_info(const rq_batch_plan* plan, rq_batch_config* cfg, int* grid,
                       long long* total_rays) {
  if (!plan) return bfail(RQ_ERR_ARG, "NULL plan");
  if (cfg) *cfg = plan->cfg;
  if (grid) *grid = plan->grid;
  if (total_rays) *total_rays = plan->total_rays;
  return RQ_OK;
}

int rq_batch_plan_destroy(rq_batch_plan* plan) {
  if (plan) {
    cudaSetDevice(plan->device);
    delete plan;
  }
  return RQ_OK;
}

int rq_batch_autotune(rq_scene* const* scenes, int n_scenes, const rq_batch* batches,
                      int n_batches, const rq_batch_config* candidates, int n_candidates,
                      int reps, rq_batch_config* best, float* best_ms) {
  if (!best) return bfail(RQ_ERR_ARG, "best is NULL");
  if (reps < 1) reps = 1;
  const rq::Scene* s0 = reinterpret_cast<const rq::Scene*>(scenes ? scenes[0] : nullptr);
  if (!s0) return bfail(RQ_ERR_ARG, "NULL scene");
  if (cudaSetDevice(s0->device) != cudaSuccess) return bfail(RQ_ERR_CUDA, "cudaSetDevice");
  cudaStream_t st;
  cudaEvent_t e0, e1;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
    return bfail(RQ_ERR_CUDA, "stream");
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float bms = 1e30f;
  int rc = RQ_OK;
  // times one configuration; keeps it if it is the fastest so far
  auto time_one = [&](const rq_batch_config& c) -> int {
    rq_batch_plan* p = nullptr;
    int r = rq_batch_plan_create(scenes, n_scenes, batches, n_batches, &c, &p);
    if (r != RQ_OK) return r;
    rq_batch_plan_launch(p, st);  // warm-up
    cudaEventRecord(e0, st);
    for (int k = 0; k < reps; ++k) rq_batch_plan_launch(p, st);
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    rq_batch_plan_destroy(p);
    if (e != cudaSuccess) return bfail(RQ_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
    ms /= reps;
    if (ms < bms) {
      bms = ms;
      *best = c;
    }
    return RQ_OK;
  };
  if (candidates && n_candidates > 0) {
    for (int i = 0; i < n_candidates && rc == RQ_OK; ++i) rc = time_one(candidates[i]);
  } else {
    // 1. launch shape, rays per warp chunk and refill (compaction)
    //    threshold, stack in shared memory, depth-first records
    for (int bt : {64, 128, 256})
      for (int cr : {32, 128, 512})
        for (int rf : {1, 8, 24}) {
          if (rc != RQ_OK) break;
          rq_batch_config c = default_batch_config();
          c.block_threads = bt;
          c.chunk_rays = cr;
          c.refill_threshold = rf;
          rc = time_one(c);
        }
    // 2. register-stack entries x node layout at the best shape
    const rq_batch_config shape = *best;
    for (int rs : {0, 1, 2, 4})
      for (int nl : {RQ_LAYOUT_DFS, RQ_LAYOUT_BFS, RQ_LAYOUT_BFS_TOP}) {
        if (rc != RQ_OK || (rs == shape.reg_stack && nl == shape.node_layout)) continue;
        rq_batch_config c = shape;
        c.reg_stack = rs;
        c.node_layout = nl;
        rc = time_one(c);
      }
    // 2b. a short shared column with a global overflow area (more resident
    //     warps) at the best shape and layout
    const rq_batch_config lay = *best;
    for (int se : {8, 12, 16}) {
      if (rc != RQ_OK) break;
      rq_batch_config c = lay;
      c.reg_stack = 0;
      c.smem_entries = se;
      rc = time_one(c);
    }
    // 3. chunk and refill again at the best stack and layout
    const rq_batch_config mid = *best;
    for (int cr : {64, 128, 256, 512})
      for (int rf : {4, 8, 16, 24}) {
        if (rc != RQ_OK || (cr == mid.chunk_rays && rf == mid.refill_threshold)) continue;
        rq_batch_config c = mid;
        c.chunk_rays = cr;
        c.refill_threshold = rf;
        rc = time_one(c);
      }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  if (rc == RQ_OK && best_ms) *best_ms = bms;
  return rc;
}

}  // extern "C"
