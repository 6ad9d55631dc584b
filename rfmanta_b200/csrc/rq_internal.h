// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "rq_device.cuh"

namespace rq {

// Device pointers of one ray batch (SoA) and its outputs.
struct RayArgs {
  int n;
  const float* org;  // 3 rows: org[c * stride + i]
  const float* dir;  // 3 rows
  const float* tmax; // n
  float* t;
  int32_t* prim;
  float* u;
  float* v;
  int stride = 0;    // elements between the rows of org/dir; 0 = n
};

struct LaunchPlan {
  int block_threads;
  int grid;         // persistent grid size
  int refill;       // idle lanes before a warp refills
  bool persistent;
  int* counter;     // device ray counter (persistent form), zeroed per launch
};

cudaError_t launch_trace(const DevScene& S, const RayArgs& a, bool anyhit,
                         const LaunchPlan& plan, cudaStream_t st);

int max_blocks_per_sm(int tri_kind, bool anyhit, bool persistent,
                      int block_threads, size_t smem);

// Writes the 48-byte triangle records in leaf order (perm[k] = original
// triangle id; bit 31 of perm[k] marks the last triangle of a leaf).
cudaError_t launch_tri_setup(int tri_kind, const float* d_verts,
                             const uint32_t* d_idx, const int32_t* d_perm,
                             int n, float4* d_tris, cudaStream_t st);

// Ordered stream compaction (rq_path.cu): the indices i < n with flags[i]
// != 0, in increasing order, into qout, and their count into *total_out;
// tile_counts holds flag_compaction_tiles(n) ints of scratch.
int flag_compaction_tiles(int n);
cudaError_t launch_flag_compaction(const uint8_t* flags, int n, int* tile_counts, int* total_out,
                                   int* qout, cudaStream_t st);

void set_error(const std::string& msg);

}  // namespace rq
