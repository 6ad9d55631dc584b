// Host-side scene object behind the opaque rq_scene handle.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_device.cuh"
#include "rq_internal.h"

namespace rq {

struct FrameScratch;
void destroy_frame(FrameScratch* f);
struct PathScratch;
void destroy_path_scratch(PathScratch* p);
struct SampleScratch;
void destroy_sample_scratch(SampleScratch* p);
struct DynTree;
void destroy_dyn_tree(DynTree* d);
struct Scene;
struct HostTree;
cudaError_t launch_trace2(const Scene& s, const RayArgs& a, bool anyhit, int32_t* inst,
                          cudaStream_t st);
int set_instance_tree(Scene* s, const HostTree& t);

// The reference DynBVH tree, field by field (Model/Groups/DynBVH.h:37-79).
struct HostTree {
  std::vector<float> bounds;  // 6 per node: min xyz, max xyz
  std::vector<int32_t> child;
  std::vector<int32_t> children;
  std::vector<uint8_t> axis;
  std::vector<uint8_t> left_cheaper;
  std::vector<int32_t> ids;  // object_ids, one per triangle
};

// DynBVH::computeCost (DynBVH.cc:3389-3416); with `costs`, every reachable
// node's cost as computeCost<true> leaves it (others 0).
double tree_sah_cost(const HostTree& t, std::vector<float>* costs = nullptr);

// A validated tree laid out for the kernels: node records (4 float4 each,
// depth-first pre-order) and the leaf-ordered object permutation (bit 31 on
// the last object of each leaf).
struct TreeLayout {
  std::vector<float4> recs;
  std::vector<int32_t> perm;
  std::vector<int32_t> rec_node;   // DynBVH node id of each record
  std::vector<int32_t> rec_depth;  // depth of each record (root = 0)
  std::vector<int32_t> rec_size;   // records in each record's subtree
  int n_records = 0;
  int n_leaves = 0;
  int root_ref = 0;
  float root_lo[3] = {0, 0, 0};
  float root_hi[3] = {0, 0, 0};
  int depth = 0;
};

int layout_tree(const HostTree& t, int n_objects, TreeLayout& out);

// Calls of up to this many rays trace straight from mapped host memory.
constexpr int kZeroCopyRays = 4096;

// Per-call resources for the host-array entry point.
struct Staging {
  cudaStream_t stream = nullptr;
  void* h_buf = nullptr;  // pinned
  void* d_buf = nullptr;
  int* d_counter = nullptr;
  size_t cap = 0;
  // small calls: pinned host memory mapped into the device's address space,
  // read and written by the kernel directly (no copies)
  void* h_map = nullptr;
  void* d_map = nullptr;
  size_t map_cap = 0;
  ~Staging();
};

struct Scene {
  int device = 0;
  int tri_kind = 0;
  int n_tris = 0;
  int n_verts = 0;
  int num_sms = 148;
  mutable std::vector<float> verts;  // host mirror; stale after a device-side update
  mutable bool verts_stale = false;
  std::vector<uint32_t> idx;
  std::vector<uint32_t> face_mat;
  int64_t max_face_material = -1;  // largest face material id (-1: no faces)
  float* d_verts = nullptr;
  uint32_t* d_idx = nullptr;
  uint32_t* d_face_mat = nullptr;

  // tree
  bool has_tree = false;
  mutable HostTree tree;      // bounds stale after a refit until refresh_tree()
  mutable bool tree_stale = false;
  // refit support: leaf-order object ids (bit 31 = last of leaf), records
  // grouped by depth (deepest level first) with level offsets, and each
  // record's DynBVH node id
  int32_t* d_perm = nullptr;
  int32_t* d_level_recs = nullptr;
  std::vector<int> level_offsets;
  std::vector<int32_t> rec_node;
  std::vector<int32_t> rec_depth;  // of the layout set_tree made
  std::vector<int32_t> rec_size;
  int rec_capacity = 0;             // records d_nodes / d_level_recs hold
  // rotating update (rq_rotate.cu): DynBVH::costs as a rebuild leaves them,
  // DynBVH::nextFree, and the device node arrays once an update has run
  std::vector<float> tree_costs;
  int tree_next_free = 0;
  DynTree* dyn = nullptr;
  mutable bool tree_from_dyn = false;  // stale host tree: read dyn, not records
  float4* d_nodes = nullptr;
  float4* d_tris = nullptr;
  float* d_root_box = nullptr;  // refit output: the root's box
  int n_records = 0;
  int n_leaves = 0;
  int n_leaf_tris = 0;
  int depth = 0;
  int root_ref = 0;
  float root_lo[3] = {0, 0, 0};
  float root_hi[3] = {0, 0, 0};

  // two-level scenes (InstanceT): the tree above is the top-level tree over
  // instances and d_tris holds 2 float4 per instance in leaf order
  // (translation xyz, inner scene index | instance id with the last-in-leaf
  // bit, kind); the inner scenes are referenced, not owned.
  bool instanced = false;
  std::vector<Scene*> blas;
  std::vector<int32_t> inst_blas;
  std::vector<float> inst_translation;
  std::vector<int32_t> inst_kind;
  DevScene* d_blas = nullptr;
  int max_blas_depth = 0;

  // bumped whenever the device tree or the descriptor dev() returns changes
  // (a new tree, an update); users that keep copies of dev() (batch plans,
  // servers, two-level scenes) compare it before they launch
  uint64_t generation = 0;
  std::vector<uint64_t> blas_generation;  // two-level: inner generations at creation
  int check_inner_current() const;

  rq_launch_config cfg[4];  // RQ_CLOSEST, RQ_ANYHIT, RQ_PATH_EXTEND, RQ_PATH_SHADE
  int* d_counter = nullptr;  // persistent-launch counters for rq_trace_device

  std::mutex mu;
  std::vector<std::unique_ptr<Staging>> staging;

  FrameScratch* frame = nullptr;  // frame-path scratch (rq_frame.cu)
  PathScratch* paths = nullptr;   // path-tracing scratch (rq_pathhost.cu)
  SampleScratch* samples = nullptr;  // supersampled-frame scratch (rq_instance.cu)
  int32_t* path_dbg_prim = nullptr;
  float* path_dbg_org = nullptr;
  float* path_dbg_dir = nullptr;
  long long path_dbg_capacity = 0;
  double last_build_seconds = 0;
  unsigned long long* stats = nullptr;  // device counters, NULL = off
  cudaEvent_t stage_events[16] = {};
  int n_stage_events = 0;
  std::mutex frame_mu;

  // resident packet channels over this scene (rq_channel.cu); their kernels
  // are stopped before the tree changes and detached when the scene goes
  std::mutex chan_mu;
  std::vector<rq_channel*> channels;

  // node records in another order (rq_layout.cu), per RQ_LAYOUT_*, made on
  // first use and kept until the tree changes
  struct AltLayout {
    float4* nodes = nullptr;
    int capacity = 0;
    int root = 0;
    uint64_t generation = ~0ull;
  };
  AltLayout alt_layout[3];
  // dev() with the records in `layout` order
  int node_layout(int layout, DevScene& out);
  void free_layouts();

  ~Scene();
  void free_tree();
  int set_tree(const HostTree& t);
  int refresh_tree() const;  // host tree bounds from the device records
  const std::vector<float>* host_vertices() const;  // NULL on a copy failure
  DevScene dev() const;
  Staging* acquire(size_t bytes_in, size_t bytes_out);
  void release(Staging* s);
  LaunchPlan plan(bool anyhit, int n, int* counter) const;
  // stride: elements between the x/y/z rows of org and dir (0 = n);
  // one_per_ray: a plain grid of one thread per ray (no work counter to
  // reset), for small batches
  int trace_device(int n, const float* org, const float* dir, const float* tmax,
                   bool anyhit, float* t, int32_t* prim, float* u, float* v,
                   cudaStream_t st, int* counter, int stride = 0, bool one_per_ray = false);
};

// Stops the kernels of the scene's channels (they start again on their next
// packet, with the scene's new descriptor); detach_channels also cuts the
// channels off the scene, which is going away.
void park_channels(Scene* s);
void detach_channels(Scene* s);

int rotate_update(Scene* s);
int sync_layout_host(Scene* s);
void mark_dyn_bounds_stale(DynTree* d);
int refresh_tree_from_dyn(const Scene* s);
int dyn_state(const Scene* s, float* costs, int cap, int* next_free);

}  // namespace rq

// The opaque handle of the C ABI is the scene itself.
struct rq_scene : public rq::Scene {};
