// Path-tracing wavefront: parameters and buffers (see rq_path.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rq_device.cuh"
#include "rq_env.cuh"

namespace rq {

constexpr int kMaxPathDepth = 16;
// counters[0..kMaxPathDepth]: live paths per depth; counters[kFetchBase + d]
// and counters[kShadeFetchBase + d]: the work counters of bounce d's
// persistent extension and shade launches
constexpr int kFetchBase = kMaxPathDepth + 1;
constexpr int kShadeFetchBase = kFetchBase + kMaxPathDepth;
constexpr int kPathCounters = kShadeFetchBase + kMaxPathDepth;

struct PathParams {
  float cam[12];  // eye, lookat-eye, u, v
  int xres, yres;
  int spp, strata;  // strata * strata == spp
  int max_depth;    // bounces (primary hit = depth 0)
  int rr_depth;     // Russian roulette from this depth on
  unsigned long long seed;
  float light_anchor[3], light_v1[3], light_v2[3];
  float light_normal[3];  // Parallelogram: unit Cross(v1, v2)
  float light_inv_area;   // 1 / |Cross(v1, v2)|
  float light_color[3];
  float background[3];
  float ambient[3];        // added at max_depth (do_ambient_on_maxdepth)
  Environment env;         // ambient and background kinds
  const float* materials;  // device, rgb per material id
};

struct PathBuffers {
  size_t capacity;      // paths per chunk
  long long g0;         // global id of the chunk's first path
  float* o;             // 3 * capacity
  float* d;
  float* imp;
  float* rad;
  unsigned long long* rng;  // PCG32 state per path
  float* t;
  int32_t* pos;
  int32_t* prim;
  int32_t* queue[2];
  int32_t* counters;            // kPathCounters (see above)
  // optional: survivor flag per path slot; when set, the next bounce's queue
  // is built in path order by an ordered compaction instead of per-warp
  // appends
  uint8_t* alive;
  int* tile_counts;  // scratch of the ordered compaction
  unsigned long long* ray_counts;  // [0] extension rays, [1] shadow rays
  unsigned long long* stats;       // optional box/tri test counters (4)
  // optional per-bounce dump for parity checks: [depth][path]
  int32_t* dbg_prim;
  float* dbg_org;  // [3][depth][path]
  float* dbg_dir;
};

// Launch shape of the two persistent bounce stages ([0] extend, [1] shade).
struct PathLaunch {
  int block_threads[2];
  int blocks_per_sm[2];  // 0 = occupancy maximum
  int refill[2];
  int reg_stack[2];      // traversal-stack entries in registers: 0, 2 or 4
};

cudaError_t launch_path_chunk(const DevScene& S, const PathParams& P, PathBuffers B,
                              long long g0, int n, float* rgb, int grid,
                              const PathLaunch& L, cudaStream_t st, const cudaEvent_t* ev,
                              int nev);
int path_blocks_per_sm(int tri_kind, size_t smem);
// Builds bounce depth+1's queue (and live count) from B.alive over slots
// [0, n), in slot order.
cudaError_t launch_ordered_compaction(const PathBuffers& B, int n, int depth, cudaStream_t st);

}  // namespace rq
