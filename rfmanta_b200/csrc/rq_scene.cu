// Scene management and the C ABI (include/rfmanta_b200.h).
//
// A scene owns, on one device:
//   * the mesh (vertices, indices, face materials) as uploaded;
//   * the node records and triangle records the kernels read;
//   * a host copy of the tree in the reference's field-wise DynBVH form
//     (for export, SAH cost and validation);
//   * a pool of staging contexts (stream + pinned and device buffers) so
//     several host threads can call rq_trace on one scene at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_device.cuh"
#include "rq_internal.h"
#include "rq_scene.h"

namespace rq {

static thread_local std::string g_error;

void set_error(const std::string& msg) { g_error = msg; }

static int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

static int cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? RQ_ERR_OOM : RQ_ERR_CUDA;
}

#define RQ_CUDA(call)                                 \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

Staging::~Staging() {
  if (stream) cudaStreamDestroy(stream);
  if (h_map) cudaFreeHost(h_map);
  if (h_buf) cudaFreeHost(h_buf);
  if (d_buf) cudaFree(d_buf);
  if (d_counter) cudaFree(d_counter);
}

Scene::~Scene() {
  detach_channels(this);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  free_tree();
  free_layouts();
  if (d_verts) cudaFree(d_verts);
  if (d_idx) cudaFree(d_idx);
  if (d_face_mat) cudaFree(d_face_mat);
  if (d_counter) cudaFree(d_counter);
  if (d_blas) cudaFree(d_blas);
  if (samples) destroy_sample_scratch(samples);
  if (frame) destroy_frame(frame);
  if (paths) destroy_path_scratch(paths);
  staging.clear();
  if (prev >= 0) cudaSetDevice(prev);
}

const std::vector<float>* Scene::host_vertices() const {
  if (verts_stale) {
    if (cudaMemcpy(verts.data(), d_verts, verts.size() * sizeof(float),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      return nullptr;
    verts_stale = false;
  }
  return &verts;
}

void Scene::free_tree() {
  if (d_root_box) cudaFree(d_root_box);
  d_root_box = nullptr;
  if (d_nodes) cudaFree(d_nodes);
  if (d_tris) cudaFree(d_tris);
  if (d_perm) cudaFree(d_perm);
  if (d_level_recs) cudaFree(d_level_recs);
  d_nodes = nullptr;
  d_tris = nullptr;
  d_perm = nullptr;
  d_level_recs = nullptr;
  level_offsets.clear();
  rec_node.clear();
  rec_depth.clear();
  rec_size.clear();
  rec_capacity = 0;
  tree_costs.clear();
  tree_next_free = 0;
  destroy_dyn_tree(dyn);
  dyn = nullptr;
  tree_from_dyn = false;
  tree_stale = false;
  has_tree = false;
}

DevScene Scene::dev() const {
  DevScene S;
  S.nodes = d_nodes;
  S.tris = d_tris;
  S.face_material = d_face_mat;
  S.tri_kind = tri_kind;
  S.root_ref = root_ref;
  for (int c = 0; c < 3; ++c) {
    S.root_lo[c] = root_lo[c];
    S.root_hi[c] = root_hi[c];
  }
  S.depth = depth > 0 ? depth : 1;
  return S;
}

// ---------------------------------------------------------------- tree ----

// Validates a field-wise DynBVH tree and lays it out as node records and a
// leaf-ordered triangle permutation.  Records are numbered in depth-first
// pre-order of the internal nodes (root = record 0), leaves' triangles are
// placed in the same pre-order, each leaf's object_ids in stored order.
int layout_tree(const HostTree& t, int n_objects, TreeLayout& L) {
  const int nn = (int)t.children.size();
  if (nn < 1) return fail(RQ_ERR_FORMAT, "tree has no nodes");
  const int nids = (int)t.ids.size();
  std::vector<int> rec_of(nn, -1);
  std::vector<int> leaf_start(nn, -1);
  std::vector<uint8_t> seen(nn, 0);
  std::vector<int32_t>& perm = L.perm;
  perm.clear();
  perm.reserve(nids);
  L.rec_depth.clear();
  std::vector<int> order;  // internal nodes in record order
  // iterative pre-order DFS; stack holds (node, depth)
  std::vector<std::pair<int, int>> st;
  st.push_back({0, 0});
  int max_depth = 0;
  while (!st.empty()) {
    const int node = st.back().first;
    const int d = st.back().second;
    st.pop_back();
    if (node < 0 || node >= nn) return fail(RQ_ERR_FORMAT, "child index out of range");
    if (seen[node]) return fail(RQ_ERR_FORMAT, "node reached twice (cycle or shared child)");
    seen[node] = 1;
    const int ch = t.children[node];
    const int c = t.child[node];
    if (ch != 0) {
      if (ch < 0 || c < 0 || (long long)c + ch > nids)
        return fail(RQ_ERR_FORMAT, "leaf object range out of bounds");
      leaf_start[node] = (int)perm.size();
      for (int i = 0; i < ch; ++i) {
        const int obj = t.ids[c + i];
        if (obj < 0 || obj >= n_objects)
          return fail(RQ_ERR_FORMAT, "object id out of range");
        perm.push_back(obj);
      }
      perm.back() |= int32_t(0x80000000u);
      max_depth = std::max(max_depth, d);
    } else {
      if (c < 0 || c + 1 >= nn) return fail(RQ_ERR_FORMAT, "internal child out of range");
      if (t.axis[node] > 2) return fail(RQ_ERR_FORMAT, "split axis out of range");
      rec_of[node] = (int)order.size();
      order.push_back(node);
      L.rec_depth.push_back(d);
      // push right first so the left subtree is laid out first
      st.push_back({c + 1, d + 1});
      st.push_back({c, d + 1});
    }
  }
  std::vector<float4>& recs = L.recs;
  recs.assign(order.size() * 4, make_float4(0.f, 0.f, 0.f, 0.f));
  auto ref_of = [&](int node) -> int {
    return t.children[node] != 0 ? ~leaf_start[node] : rec_of[node];
  };
  for (size_t r = 0; r < order.size(); ++r) {
    const int node = order[r];
    const int L = t.child[node], R = L + 1;
    const float* bl = &t.bounds[6 * (size_t)L];
    const float* br = &t.bounds[6 * (size_t)R];
    recs[4 * r + 0] = make_float4(bl[0], bl[1], bl[2], bl[3]);
    recs[4 * r + 1] = make_float4(bl[4], bl[5], br[0], br[1]);
    recs[4 * r + 2] = make_float4(br[2], br[3], br[4], br[5]);
    const int meta = (t.axis[node] & 3) | ((t.left_cheaper[node] & 1) << 2);
    int4 q3 = make_int4(ref_of(L), ref_of(R), meta, 0);
    std::memcpy(&recs[4 * r + 3], &q3, sizeof(q3));
  }
  L.rec_node = order;
  L.n_records = (int)order.size();
  // subtree record counts: children come after their parent in pre-order
  L.rec_size.assign(order.size(), 1);
  for (size_t r = order.size(); r-- > 0;) {
    int4 q3;
    std::memcpy(&q3, &recs[4 * r + 3], sizeof(q3));
    if (q3.x >= 0) L.rec_size[r] += L.rec_size[q3.x];
    if (q3.y >= 0) L.rec_size[r] += L.rec_size[q3.y];
  }
  L.n_leaves = 0;
  for (int i = 0; i < nn; ++i)
    if (seen[i] && t.children[i] != 0) ++L.n_leaves;
  L.root_ref = ref_of(0);
  for (int c = 0; c < 3; ++c) {
    L.root_lo[c] = t.bounds[c];
    L.root_hi[c] = t.bounds[3 + c];
  }
  L.depth = max_depth;
  if (L.depth > kMaxDepth)
    return fail(RQ_ERR_CAPACITY, "tree depth " + std::to_string(L.depth) +
                                     " exceeds the traversal stack limit");
  return RQ_OK;
}

int Scene::set_tree(const HostTree& t) {
  if (instanced) return set_instance_tree(this, t);
  park_channels(this);
  TreeLayout L;
  const int rc = layout_tree(t, n_tris, L);
  if (rc != RQ_OK) return rc;
  const std::vector<float4>& recs = L.recs;
  const std::vector<int32_t>& perm = L.perm;
  // device upload
  free_tree();
  const size_t rec_bytes = std::max<size_t>(recs.size(), 4) * sizeof(float4);
  const size_t tri_bytes = std::max<size_t>(perm.size(), 1) * 3 * sizeof(float4);
  RQ_CUDA(cudaMalloc(&d_nodes, rec_bytes));
  RQ_CUDA(cudaMalloc(&d_tris, tri_bytes));
  if (!recs.empty())
    RQ_CUDA(cudaMemcpy(d_nodes, recs.data(), recs.size() * sizeof(float4),
                       cudaMemcpyHostToDevice));
  RQ_CUDA(cudaMalloc(&d_perm, std::max<size_t>(perm.size(), 1) * sizeof(int32_t)));
  cudaError_t e = cudaMemcpy(d_perm, perm.data(), perm.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = launch_tri_setup(tri_kind, d_verts, d_idx, d_perm, (int)perm.size(),
                         d_tris, 0);
  // records grouped by depth, deepest first (the refit's bottom-up order)
  const int nrec = L.n_records;
  std::vector<int32_t> by_level(nrec);
  level_offsets.assign(1, 0);
  if (nrec > 0) {
    int maxd = 0;
    for (int d : L.rec_depth) maxd = std::max(maxd, d);
    std::vector<int> count(maxd + 1, 0);
    for (int d : L.rec_depth) ++count[d];
    std::vector<int> start(maxd + 2, 0);
    for (int d = maxd; d >= 0; --d) start[maxd - d + 1] = start[maxd - d] + count[d];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int r = 0; r < nrec; ++r) by_level[fill[maxd - L.rec_depth[r]]++] = r;
    level_offsets.assign(start.begin(), start.end());
  }
  if (e == cudaSuccess) e = cudaMalloc(&d_level_recs, std::max(nrec, 1) * sizeof(int32_t));
  if (e == cudaSuccess && nrec > 0)
    e = cudaMemcpy(d_level_recs, by_level.data(), nrec * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "triangle setup");
  rec_node = L.rec_node;
  rec_depth = L.rec_depth;
  rec_size = L.rec_size;
  rec_capacity = L.n_records;
  tree = t;
  tree_sah_cost(t, &tree_costs);
  tree_next_free = (int)t.children.size();
  n_records = L.n_records;
  n_leaf_tris = (int)perm.size();
  n_leaves = L.n_leaves;
  root_ref = L.root_ref;
  for (int c = 0; c < 3; ++c) {
    root_lo[c] = L.root_lo[c];
    root_hi[c] = L.root_hi[c];
  }
  depth = L.depth;
  has_tree = true;
  ++generation;
  return RQ_OK;
}

int Scene::check_inner_current() const {
  for (size_t i = 0; i < blas.size(); ++i)
    if (i >= blas_generation.size() || blas[i]->generation != blas_generation[i])
      return fail(RQ_ERR_STATE, "an inner scene changed after the two-level scene was made; "
                                "create the two-level scene again");
  return RQ_OK;
}

// BBox::computeArea (Core/Geometry/BBox.h:117-121), evaluated in float.
static float box_area(const float* b) {
  const volatile float dx = b[3] - b[0];
  const volatile float dy = b[4] - b[1];
  const volatile float dz = b[5] - b[2];
  const volatile float xy = dx * dy;
  const volatile float yz = dy * dz;
  const volatile float xz = dx * dz;
  const volatile float s1 = xy + yz;
  const volatile float s2 = s1 + xz;
  return 2 * s2;
}

// DynBVH::computeCost (DynBVH.cc:3389-3416) with C_isec = C_trav = 1,
// bottom-up over the pre-order so no recursion is needed.
double tree_sah_cost(const HostTree& t, std::vector<float>* costs) {
  const int nn = (int)t.children.size();
  std::vector<int> order;
  std::vector<int> st(1, 0);
  while (!st.empty()) {
    const int n = st.back();
    st.pop_back();
    order.push_back(n);
    if (t.children[n] == 0) {
      st.push_back(t.child[n]);
      st.push_back(t.child[n] + 1);
    }
  }
  std::vector<float> cost(nn, 0.f);
  for (size_t k = order.size(); k-- > 0;) {
    const int n = order[k];
    if (t.children[n] != 0) {
      cost[n] = t.children[n] * 1.f;
    } else {
      const int L = t.child[n], R = L + 1;
      const float area = box_area(&t.bounds[6 * (size_t)n]);
      const float la = box_area(&t.bounds[6 * (size_t)L]);
      const float ra = box_area(&t.bounds[6 * (size_t)R]);
      const volatile float a = la * cost[L];
      const volatile float b = ra * cost[R];
      const volatile float s = a + b;
      const volatile float q = s / area;
      cost[n] = 1.f + q;
    }
  }
  if (costs) *costs = cost;
  return cost[0];
}

// ----------------------------------------------------------- staging ----

Staging* Scene::acquire(size_t bytes_in, size_t bytes_out) {
  std::unique_ptr<Staging> s;
  {
    std::lock_guard<std::mutex> g(mu);
    if (!staging.empty()) {
      s = std::move(staging.back());
      staging.pop_back();
    }
  }
  if (!s) {
    s.reset(new Staging());
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
      return nullptr;
    if (cudaMalloc(&s->d_counter, sizeof(int)) != cudaSuccess) return nullptr;
  }
  const size_t need = bytes_in + bytes_out;
  if (s->cap < need) {
    if (s->h_buf) cudaFreeHost(s->h_buf);
    if (s->d_buf) cudaFree(s->d_buf);
    s->h_buf = nullptr;
    s->d_buf = nullptr;
    size_t cap = std::max<size_t>(need, 1 << 16);
    if (cudaMallocHost(&s->h_buf, cap) != cudaSuccess) return nullptr;
    if (cudaMalloc(&s->d_buf, cap) != cudaSuccess) return nullptr;
    s->cap = cap;
  }
  return s.release();
}

void Scene::release(Staging* s) {
  std::lock_guard<std::mutex> g(mu);
  staging.emplace_back(s);
}

LaunchPlan Scene::plan(bool anyhit, int n, int* counter) const {
  const rq_launch_config& c = cfg[anyhit ? 1 : 0];
  LaunchPlan p;
  p.block_threads = c.block_threads;
  p.persistent = c.persistent != 0 && n > 0;
  p.refill = std::max(1, std::min(32, c.refill_threshold));
  p.counter = counter;
  int bps = c.blocks_per_sm;
  const size_t smem = (size_t)std::max(depth, 1) * c.block_threads * sizeof(int2);
  if (bps <= 0)
    bps = max_blocks_per_sm(tri_kind, anyhit, p.persistent, c.block_threads, smem);
  else
    max_blocks_per_sm(tri_kind, anyhit, p.persistent, c.block_threads, smem);
  p.grid = std::max(1, bps * num_sms);
  // never launch more persistent threads than rays
  const int need_blocks = (n + c.block_threads - 1) / c.block_threads;
  if (p.persistent && p.grid > need_blocks) p.grid = std::max(1, need_blocks);
  return p;
}

int Scene::trace_device(int n, const float* org, const float* dir,
                        const float* tmax, bool anyhit, float* t, int32_t* prim,
                        float* u, float* v, cudaStream_t st, int* counter, int stride,
                        bool one_per_ray) {
  if (!has_tree) return fail(RQ_ERR_STATE, "scene has no tree");
  if (instanced) {
    const int rc = check_inner_current();
    if (rc != RQ_OK) return rc;
  }
  RayArgs a{n, org, dir, tmax, t, prim, u, v, stride};
  LaunchPlan p;
  if (one_per_ray) {
    // a plain grid sized by the launch itself: no work counter, and no
    // occupancy query on this per-packet path
    const rq_launch_config& c = cfg[anyhit ? 1 : 0];
    p.block_threads = c.block_threads;
    p.grid = 1;
    p.refill = 1;
    p.persistent = false;
    p.counter = nullptr;
    const size_t smem = (size_t)std::max(depth, 1) * c.block_threads * sizeof(int2);
    if (smem > 48 * 1024) max_blocks_per_sm(tri_kind, anyhit, false, c.block_threads, smem);
  } else {
    p = plan(anyhit, n, counter);
  }
  if (p.persistent) {
    if (!counter) return fail(RQ_ERR_ARG, "persistent launch needs a counter");
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  }
  cudaError_t e = instanced ? launch_trace2(*this, a, anyhit, nullptr, st)
                            : launch_trace(dev(), a, anyhit, p, st);
  if (e != cudaSuccess) return cuda_fail(e, "trace launch");
  return RQ_OK;
}

}  // namespace rq

// ==================================================================== ABI ==

using rq::fail;
using rq::cuda_fail;

extern "C" {

const char* rq_last_error(void) { return rq::g_error.c_str(); }

const char* rq_version(void) { return "rfmanta_b200 0.1.0 sm_100a"; }

int rq_scene_create(const float* vertices, int n_vertices,
                    const uint32_t* indices, int n_tris,
                    const uint32_t* face_material, int tri_kind, int device,
                    rq_scene** out) {
  if (!out) return fail(RQ_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!vertices || !indices || n_vertices <= 0 || n_tris <= 0)
    return fail(RQ_ERR_ARG, "empty or NULL mesh");
  if (tri_kind != RQ_TRI_WALD && tri_kind != RQ_TRI_KS)
    return fail(RQ_ERR_ARG, "unknown triangle kind");
  for (long long i = 0; i < 3LL * n_tris; ++i)
    if (indices[i] >= (uint32_t)n_vertices)
      return fail(RQ_ERR_ARG, "vertex index out of range");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
    return fail(RQ_ERR_NODEV, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(RQ_ERR_ARG, "bad device ordinal");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10)
    return fail(RQ_ERR_NODEV, "device is not sm_100 class");
  std::unique_ptr<rq_scene> s(new rq_scene());
  s->device = device;
  s->tri_kind = tri_kind;
  s->n_tris = n_tris;
  s->n_verts = n_vertices;
  s->num_sms = prop.multiProcessorCount;
  s->verts.assign(vertices, vertices + 3 * (size_t)n_vertices);
  s->idx.assign(indices, indices + 3 * (size_t)n_tris);
  if (face_material)
    s->face_mat.assign(face_material, face_material + n_tris);
  else
    s->face_mat.assign(n_tris, 0u);
  for (uint32_t m : s->face_mat) s->max_face_material = std::max<int64_t>(s->max_face_material, m);
  RQ_CUDA(cudaSetDevice(device));
  RQ_CUDA(cudaMalloc(&s->d_verts, s->verts.size() * sizeof(float)));
  RQ_CUDA(cudaMalloc(&s->d_idx, s->idx.size() * sizeof(uint32_t)));
  RQ_CUDA(cudaMalloc(&s->d_face_mat, s->face_mat.size() * sizeof(uint32_t)));
  RQ_CUDA(cudaMemcpy(s->d_verts, s->verts.data(), s->verts.size() * sizeof(float),
                     cudaMemcpyHostToDevice));
  RQ_CUDA(cudaMemcpy(s->d_idx, s->idx.data(), s->idx.size() * sizeof(uint32_t),
                     cudaMemcpyHostToDevice));
  RQ_CUDA(cudaMemcpy(s->d_face_mat, s->face_mat.data(),
                     s->face_mat.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  for (int k = 0; k < 4; ++k) {
    s->cfg[k].block_threads = 128;
    s->cfg[k].blocks_per_sm = 0;
    s->cfg[k].refill_threshold = 8;
    s->cfg[k].persistent = 1;
    s->cfg[k].reg_stack = 0;
    s->cfg[k].node_layout = RQ_LAYOUT_DFS;
  }
  // path stages: refill thresholds from a sweep of the 1280x720x16 path
  // frame (block 64/128/256 x refill 4..24)
  s->cfg[RQ_PATH_EXTEND].refill_threshold = 16;
  s->cfg[RQ_PATH_SHADE].refill_threshold = 24;
  *out = s.release();
  return RQ_OK;
}

int rq_scene_destroy(rq_scene* scene) {
  delete scene;
  return RQ_OK;
}

int rq_scene_import_tree(rq_scene* s, int n_nodes, const float* bounds,
                         const int32_t* child, const int32_t* children,
                         const uint8_t* axis, const uint8_t* left_cheaper,
                         const int32_t* object_ids) {
  if (!s || n_nodes <= 0 || !bounds || !child || !children || !axis ||
      !object_ids)
    return fail(RQ_ERR_ARG, "bad tree arguments");
  RQ_CUDA(cudaSetDevice(s->device));
  rq::HostTree t;
  t.bounds.assign(bounds, bounds + 6 * (size_t)n_nodes);
  t.child.assign(child, child + n_nodes);
  t.children.assign(children, children + n_nodes);
  t.axis.assign(axis, axis + n_nodes);
  if (left_cheaper)
    t.left_cheaper.assign(left_cheaper, left_cheaper + n_nodes);
  else
    t.left_cheaper.assign(n_nodes, 0);
  // object_ids has one entry per triangle (DynBVH::allocate, DynBVH.cc:1683)
  t.ids.assign(object_ids, object_ids + s->n_tris);
  return s->set_tree(t);
}

int rq_scene_import_dynbvh(rq_scene* s, const void* blob, size_t bytes) {
  if (!s || !blob) return fail(RQ_ERR_ARG, "NULL argument");
  const unsigned char* p = static_cast<const unsigned char*>(blob);
  size_t off = 0;
  auto take = [&](void* dst, size_t n) -> bool {
    if (off + n > bytes) return false;
    std::memcpy(dst, p + off, n);
    off += n;
    return true;
  };
  uint32_t nids = 0, nnodes = 0;
  if (!take(&nids, 4)) return fail(RQ_ERR_FORMAT, "truncated blob (ids count)");
  if ((size_t)nids * 4 > bytes) return fail(RQ_ERR_FORMAT, "truncated blob (ids)");
  rq::HostTree t;
  t.ids.resize(nids);
  if (!take(t.ids.data(), (size_t)nids * 4)) return fail(RQ_ERR_FORMAT, "truncated blob (ids)");
  if (!take(&nnodes, 4)) return fail(RQ_ERR_FORMAT, "truncated blob (node count)");
  if ((size_t)nnodes * 32 > bytes - off) return fail(RQ_ERR_FORMAT, "truncated blob (nodes)");
  if (nnodes == 0) return fail(RQ_ERR_FORMAT, "blob has no nodes");
  if ((int)nids < s->n_tris) return fail(RQ_ERR_FORMAT, "blob has fewer object ids than triangles");
  t.bounds.resize(6 * (size_t)nnodes);
  t.child.resize(nnodes);
  t.children.resize(nnodes);
  t.axis.resize(nnodes);
  t.left_cheaper.resize(nnodes);
  for (uint32_t i = 0; i < nnodes; ++i) {
    const unsigned char* q = p + off + 32 * (size_t)i;
    std::memcpy(&t.bounds[6 * (size_t)i], q, 24);
    std::memcpy(&t.child[i], q + 24, 4);
    t.axis[i] = q[28];
    t.left_cheaper[i] = q[29] & 1;
    int16_t ch;
    std::memcpy(&ch, q + 30, 2);
    t.children[i] = ch;
  }
  t.ids.resize(s->n_tris);
  RQ_CUDA(cudaSetDevice(s->device));
  return s->set_tree(t);
}

int rq_scene_export_dynbvh(const rq_scene* s, void* blob, size_t* bytes) {
  if (!s || !bytes) return fail(RQ_ERR_ARG, "NULL argument");
  if (!s->has_tree) return fail(RQ_ERR_STATE, "scene has no tree");
  const int rc = s->refresh_tree();
  if (rc != RQ_OK) return rc;
  const rq::HostTree& t = s->tree;
  const uint32_t nids = (uint32_t)t.ids.size();
  const uint32_t nn = (uint32_t)t.children.size();
  const size_t need = 4 + 4 * (size_t)nids + 4 + 32 * (size_t)nn;
  if (!blob) {
    *bytes = need;
    return RQ_OK;
  }
  if (*bytes < need) return fail(RQ_ERR_ARG, "blob buffer too small");
  unsigned char* p = static_cast<unsigned char*>(blob);
  std::memcpy(p, &nids, 4);
  std::memcpy(p + 4, t.ids.data(), 4 * (size_t)nids);
  size_t off = 4 + 4 * (size_t)nids;
  std::memcpy(p + off, &nn, 4);
  off += 4;
  for (uint32_t i = 0; i < nn; ++i) {
    unsigned char* q = p + off + 32 * (size_t)i;
    std::memset(q, 0, 32);
    std::memcpy(q, &t.bounds[6 * (size_t)i], 24);
    std::memcpy(q + 24, &t.child[i], 4);
    q[28] = t.axis[i];
    q[29] = t.left_cheaper[i] & 1;
    int16_t ch = (int16_t)t.children[i];
    std::memcpy(q + 30, &ch, 2);
  }
  *bytes = need;
  return RQ_OK;
}

int rq_scene_sah_cost(const rq_scene* s, double* cost) {
  if (!s || !cost) return fail(RQ_ERR_ARG, "NULL argument");
  if (!s->has_tree) return fail(RQ_ERR_STATE, "scene has no tree");
  const int rc = s->refresh_tree();
  if (rc != RQ_OK) return rc;
  *cost = rq::tree_sah_cost(s->tree);
  return RQ_OK;
}

int rq_scene_info(const rq_scene* s, int* n_records, int* n_leaves, int* depth,
                  size_t* device_bytes) {
  if (!s) return fail(RQ_ERR_ARG, "NULL scene");
  if (n_records) *n_records = s->n_records;
  if (n_leaves) *n_leaves = s->n_leaves;
  if (depth) *depth = s->depth;
  if (device_bytes)
    *device_bytes = (size_t)s->n_records * 64 + (size_t)s->n_leaf_tris * 48 +
                    s->verts.size() * 4 + s->idx.size() * 4 + s->face_mat.size() * 4;
  return RQ_OK;
}

int rq_trace_device(rq_scene* s, int n, const float* d_org, const float* d_dir,
                    const float* d_tmax, int flags, float* d_t, int32_t* d_prim,
                    float* d_u, float* d_v, void* stream) {
  if (!s) return fail(RQ_ERR_ARG, "NULL scene");
  if (n < 0 || (n > 0 && (!d_org || !d_dir || !d_tmax)))
    return fail(RQ_ERR_ARG, "bad ray arrays");
  if (flags != RQ_CLOSEST && flags != RQ_ANYHIT) return fail(RQ_ERR_ARG, "bad flags");
  if (n == 0) return RQ_OK;
  RQ_CUDA(cudaSetDevice(s->device));
  if (!s->d_counter) RQ_CUDA(cudaMalloc(&s->d_counter, 2 * sizeof(int)));
  return s->trace_device(n, d_org, d_dir, d_tmax, flags == RQ_ANYHIT, d_t, d_prim,
                         d_u, d_v, static_cast<cudaStream_t>(stream),
                         s->d_counter + (flags == RQ_ANYHIT ? 1 : 0));
}

int rq_trace(rq_scene* s, int n, const float* org, const float* dir,
             const float* tmax, int flags, float* t, int32_t* prim, float* u,
             float* v) {
  if (!s) return fail(RQ_ERR_ARG, "NULL scene");
  if (n < 0 || (n > 0 && (!org || !dir || !tmax)))
    return fail(RQ_ERR_ARG, "bad ray arrays");
  if (flags != RQ_CLOSEST && flags != RQ_ANYHIT) return fail(RQ_ERR_ARG, "bad flags");
  if (n == 0) return RQ_OK;
  if (!s->has_tree) return fail(RQ_ERR_STATE, "scene has no tree");
  RQ_CUDA(cudaSetDevice(s->device));
  const size_t in_bytes = 7 * (size_t)n * sizeof(float);
  const size_t out_bytes = 4 * (size_t)n * sizeof(float);
  rq::Staging* st = s->acquire(in_bytes, out_bytes);
  if (!st) return fail(RQ_ERR_OOM, "staging allocation failed");
  if (n <= rq::kZeroCopyRays) {
    // a packet-sized call: the kernel reads the rays from, and writes the
    // hits to, mapped pinned host memory; one launch and one synchronise
    if (!st->h_map) {
      const size_t cap = 11 * (size_t)rq::kZeroCopyRays * sizeof(float);
      if (cudaHostAlloc(&st->h_map, cap, cudaHostAllocMapped) != cudaSuccess ||
          cudaHostGetDevicePointer(&st->d_map, st->h_map, 0) != cudaSuccess) {
        s->release(st);
        return fail(RQ_ERR_OOM, "mapped staging allocation failed");
      }
      st->map_cap = cap;
    }
    float* h = static_cast<float*>(st->h_map);
    std::memcpy(h, org, 3 * (size_t)n * sizeof(float));
    std::memcpy(h + 3 * (size_t)n, dir, 3 * (size_t)n * sizeof(float));
    std::memcpy(h + 6 * (size_t)n, tmax, (size_t)n * sizeof(float));
    float* d = static_cast<float*>(st->d_map);
    float* d_out = d + 7 * (size_t)n;
    int rc = s->trace_device(n, d, d + 3 * (size_t)n, d + 6 * (size_t)n, flags == RQ_ANYHIT,
                             d_out, reinterpret_cast<int32_t*>(d_out + n), d_out + 2 * (size_t)n,
                             d_out + 3 * (size_t)n, st->stream, st->d_counter, 0, true);
    if (rc == RQ_OK) {
      const cudaError_t e = cudaStreamSynchronize(st->stream);
      if (e != cudaSuccess) rc = cuda_fail(e, "trace");
    }
    if (rc == RQ_OK) {
      const float* o = h + 7 * (size_t)n;
      if (t) std::memcpy(t, o, (size_t)n * sizeof(float));
      if (prim) std::memcpy(prim, o + n, (size_t)n * sizeof(int32_t));
      if (u) std::memcpy(u, o + 2 * (size_t)n, (size_t)n * sizeof(float));
      if (v) std::memcpy(v, o + 3 * (size_t)n, (size_t)n * sizeof(float));
    }
    s->release(st);
    return rc;
  }
  float* h = static_cast<float*>(st->h_buf);
  std::memcpy(h, org, 3 * (size_t)n * sizeof(float));
  std::memcpy(h + 3 * (size_t)n, dir, 3 * (size_t)n * sizeof(float));
  std::memcpy(h + 6 * (size_t)n, tmax, (size_t)n * sizeof(float));
  float* d = static_cast<float*>(st->d_buf);
  float* d_out = d + 7 * (size_t)n;
  int rc = RQ_OK;
  cudaError_t e = cudaMemcpyAsync(d, h, in_bytes, cudaMemcpyHostToDevice, st->stream);
  if (e != cudaSuccess) rc = cuda_fail(e, "H2D");
  if (rc == RQ_OK)
    rc = s->trace_device(n, d, d + 3 * (size_t)n, d + 6 * (size_t)n, flags == RQ_ANYHIT,
                         d_out, reinterpret_cast<int32_t*>(d_out + n), d_out + 2 * (size_t)n,
                         d_out + 3 * (size_t)n, st->stream, st->d_counter);
  float* h_out = h + 7 * (size_t)n;
  if (rc == RQ_OK) {
    e = cudaMemcpyAsync(h_out, d_out, out_bytes, cudaMemcpyDeviceToHost, st->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st->stream);
    if (e != cudaSuccess) rc = cuda_fail(e, "D2H");
  }
  if (rc == RQ_OK) {
    if (t) std::memcpy(t, h_out, (size_t)n * sizeof(float));
    if (prim) std::memcpy(prim, h_out + n, (size_t)n * sizeof(int32_t));
    if (u) std::memcpy(u, h_out + 2 * (size_t)n, (size_t)n * sizeof(float));
    if (v) std::memcpy(v, h_out + 3 * (size_t)n, (size_t)n * sizeof(float));
  }
  s->release(st);
  return rc;
}

int rq_set_stats(rq_scene* s, uint64_t* d_counters) {
  if (!s) return fail(RQ_ERR_ARG, "NULL scene");
  s->stats = reinterpret_cast<unsigned long long*>(d_counters);
  return RQ_OK;
}

int rq_scene_build_seconds(const rq_scene* s, double* seconds) {
  if (!s || !seconds) return fail(RQ_ERR_ARG, "NULL argument");
  *seconds = s->last_build_seconds;
  return RQ_OK;
}

int rq_set_stage_events(rq_scene* s, void* events, int n) {
  if (!s || n < 0 || n > 16 || (n > 0 && !events)) return fail(RQ_ERR_ARG, "0..16 events");
  s->n_stage_events = n;
  for (int i = 0; i < n; ++i) s->stage_events[i] = static_cast<cudaEvent_t*>(events)[i];
  return RQ_OK;
}

int rq_set_launch_config(rq_scene* s, int flags, const rq_launch_config* cfg) {
  if (!s || !cfg) return fail(RQ_ERR_ARG, "NULL argument");
  if (flags < RQ_CLOSEST || flags > RQ_PATH_SHADE) return fail(RQ_ERR_ARG, "bad flags");
  if (cfg->block_threads < 32 || cfg->block_threads > 256 || cfg->block_threads % 32)
    return fail(RQ_ERR_ARG, "block_threads must be a multiple of 32 in [32, 256]");
  if (cfg->blocks_per_sm < 0 || cfg->blocks_per_sm > 64)
    return fail(RQ_ERR_ARG, "blocks_per_sm out of range");
  if (cfg->refill_threshold < 1 || cfg->refill_threshold > 32)
    return fail(RQ_ERR_ARG, "refill_threshold must be in [1, 32]");
  if (cfg->reg_stack < 0 || cfg->reg_stack > 4 || cfg->reg_stack == 3)
    return fail(RQ_ERR_ARG, "reg_stack must be 0, 1, 2 or 4");
  if (cfg->node_layout < RQ_LAYOUT_DFS || cfg->node_layout > RQ_LAYOUT_BFS_TOP)
    return fail(RQ_ERR_ARG, "node_layout must be one of RQ_LAYOUT_*");
  s->cfg[flags] = *cfg;
  return RQ_OK;
}

int rq_get_launch_config(const rq_scene* s, int flags, rq_launch_config* cfg) {
  if (!s || !cfg) return fail(RQ_ERR_ARG, "NULL argument");
  if (flags < RQ_CLOSEST || flags > RQ_PATH_SHADE) return fail(RQ_ERR_ARG, "bad flags");
  *cfg = s->cfg[flags];
  return RQ_OK;
}

}  // extern "C"
