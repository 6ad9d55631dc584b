// Refit after the mesh moved (rq_scene_update_vertices): the reference's
// DynBVH::update (Model/Groups/DynBVH.cc:1574-1581, parallelUpdateBounds
// and updateBounds 2012-2123) keeps the tree's topology and recomputes
// every node's bounds bottom up - a leaf's box is the union of its
// triangles' vertex boxes (MeshTriangle::computeBounds -> Mesh::getBBox), an
// internal node's the union of its two children - after the triangles have
// re-run their precomputation from the new vertices (WaldTriangle::update,
// WaldTriangle.cc:17-25).
//
// Here: the new vertices are uploaded, the triangle records are rebuilt in
// leaf order by the same setup kernels as a fresh tree, and the node records
// (each holding its two children's boxes) are refitted one tree level per
// launch, deepest level first, one thread per record.  Min and max are
// exact, so the boxes are bit-identical to the reference's whatever the
// order of the unions.  The host copy of the tree is refreshed from the
// records only when it is read (export, SAH cost).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_internal.h"
#include "rq_scene.h"

namespace rq {

__device__ __forceinline__ void leaf_box(const float* __restrict__ verts,
                                         const uint32_t* __restrict__ idx,
                                         const int32_t* __restrict__ perm, int first,
                                         float* lo, float* hi) {
  bool init = false;
  for (int j = first;; ++j) {
    const int tag = __ldg(perm + j);
    const int obj = tag & 0x7fffffff;
    for (int k = 0; k < 3; ++k) {
      const float* p = verts + 3 * (size_t)__ldg(idx + 3 * (size_t)obj + k);
      for (int c = 0; c < 3; ++c) {
        const float x = __ldg(p + c);
        // BBox::extendByPoint / extendByBox: Min(a, b) = a < b ? a : b
        lo[c] = init ? (lo[c] < x ? lo[c] : x) : x;
        hi[c] = init ? (hi[c] > x ? hi[c] : x) : x;
      }
      init = true;
    }
    if (tag < 0) break;  // last triangle of the leaf
  }
}

__device__ __forceinline__ void child_box(const float4* nodes, const float* verts,
                                          const uint32_t* idx, const int32_t* perm, int ref,
                                          float* lo, float* hi) {
  if (ref < 0) {
    leaf_box(verts, idx, perm, ~ref, lo, hi);
    return;
  }
  const float4* p = nodes + 4 * (size_t)ref;
  const float4 q0 = p[0], q1 = p[1], q2 = p[2];
  // reset, extendByBox(left), extendByBox(right) with the reference's Min/Max
  lo[0] = q0.x < q1.z ? q0.x : q1.z;
  lo[1] = q0.y < q1.w ? q0.y : q1.w;
  lo[2] = q0.z < q2.x ? q0.z : q2.x;
  hi[0] = q0.w > q2.y ? q0.w : q2.y;
  hi[1] = q1.x > q2.z ? q1.x : q2.z;
  hi[2] = q1.y > q2.w ? q1.y : q2.w;
}

__global__ void refit_level_kernel(float4* nodes, const int32_t* __restrict__ level_recs,
                                   int n, const float* __restrict__ verts,
                                   const uint32_t* __restrict__ idx,
                                   const int32_t* __restrict__ perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = __ldg(level_recs + i);
  float4* p = nodes + 4 * (size_t)r;
  const int4 q3 = reinterpret_cast<const int4*>(p)[3];
  float l0[3], l1[3], r0[3], r1[3];
  child_box(nodes, verts, idx, perm, q3.x, l0, l1);
  child_box(nodes, verts, idx, perm, q3.y, r0, r1);
  p[0] = make_float4(l0[0], l0[1], l0[2], l1[0]);
  p[1] = make_float4(l1[1], l1[2], r0[0], r0[1]);
  p[2] = make_float4(r0[2], r1[0], r1[1], r1[2]);
}

// Root box (DynBVH::updateBounds(0)) into out[6].
__global__ void refit_root_kernel(const float4* nodes, int root_ref, const float* verts,
                                  const uint32_t* idx, const int32_t* perm, float* out) {
  float lo[3], hi[3];
  if (root_ref < 0) {
    leaf_box(verts, idx, perm, ~root_ref, lo, hi);
  } else {
    child_box(nodes, verts, idx, perm, root_ref, lo, hi);
  }
  for (int c = 0; c < 3; ++c) {
    out[c] = lo[c];
    out[3 + c] = hi[c];
  }
}

int Scene::refresh_tree() const {
  if (!tree_stale) return RQ_OK;
  if (tree_from_dyn) {
    const int rc = refresh_tree_from_dyn(this);
    if (rc != RQ_OK) return rc;
    tree_from_dyn = false;
    tree_stale = false;
    return RQ_OK;
  }
  std::vector<float4> recs((size_t)n_records * 4);
  if (n_records > 0 &&
      cudaMemcpy(recs.data(), d_nodes, recs.size() * sizeof(float4), cudaMemcpyDeviceToHost) !=
          cudaSuccess) {
    set_error("reading refitted node records");
    return RQ_ERR_CUDA;
  }
  HostTree& t = tree;
  for (int r = 0; r < n_records; ++r) {
    const int node = rec_node[r];
    const int L = t.child[node];
    const float* q = reinterpret_cast<const float*>(&recs[4 * (size_t)r]);
    float* bl = &t.bounds[6 * (size_t)L];
    float* br = &t.bounds[6 * (size_t)(L + 1)];
    for (int k = 0; k < 6; ++k) {
      bl[k] = q[k];
      br[k] = q[6 + k];
    }
    // updateBounds sets a leaf's axis to 0
    if (t.children[L] != 0) t.axis[L] = 0;
    if (t.children[L + 1] != 0) t.axis[L + 1] = 0;
  }
  for (int c = 0; c < 3; ++c) {
    t.bounds[c] = root_lo[c];
    t.bounds[3 + c] = root_hi[c];
  }
  if (t.children[0] != 0) t.axis[0] = 0;
  tree_stale = false;
  return RQ_OK;
}

}  // namespace rq

namespace rq {
namespace {

// The update after the new positions are in the scene's device vertices.
int update_tree(Scene* s, int mode) {
  if (mode == RQ_UPDATE_ROTATE) return rotate_update(s);
  cudaError_t e = launch_tri_setup(s->tri_kind, s->d_verts, s->d_idx, s->d_perm,
                                   s->n_leaf_tris, s->d_tris, 0);
  const int nlev = (int)s->level_offsets.size() - 1;
  for (int k = 0; e == cudaSuccess && k < nlev; ++k) {
    const int a = s->level_offsets[k], n = s->level_offsets[k + 1] - a;
    if (n <= 0) continue;
    refit_level_kernel<<<(n + 127) / 128, 128>>>(s->d_nodes, s->d_level_recs + a, n,
                                                 s->d_verts, s->d_idx, s->d_perm);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && !s->d_root_box) e = cudaMalloc(&s->d_root_box, 6 * sizeof(float));
  if (e == cudaSuccess) {
    refit_root_kernel<<<1, 1>>>(s->d_nodes, s->root_ref, s->d_verts, s->d_idx, s->d_perm,
                                s->d_root_box);
    e = cudaGetLastError();
  }
  float root[6];
  if (e == cudaSuccess)
    e = cudaMemcpy(root, s->d_root_box, sizeof(root), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    set_error(std::string("refit: ") + cudaGetErrorString(e));
    return RQ_ERR_CUDA;
  }
  for (int c = 0; c < 3; ++c) {
    s->root_lo[c] = root[c];
    s->root_hi[c] = root[3 + c];
  }
  s->tree_stale = true;
  s->tree_from_dyn = false;
  if (s->dyn) mark_dyn_bounds_stale(s->dyn);
  ++s->generation;
  return RQ_OK;
}

// Argument and state checks shared by both entry points; takes the lock
// and brings the host tree up to date where a refit needs it.
int update_begin(Scene* s, const void* vertices, int n_vertices, int mode) {
  if (!s || !vertices) {
    set_error("NULL argument");
    return RQ_ERR_ARG;
  }
  park_channels(s);
  if (mode != RQ_UPDATE_REFIT && mode != RQ_UPDATE_ROTATE) {
    set_error("unknown update mode");
    return RQ_ERR_ARG;
  }
  if (s->instanced) {
    set_error("update the inner scenes of a two-level scene and create it again");
    return RQ_ERR_ARG;
  }
  if (n_vertices != s->n_verts) {
    set_error("vertex count differs from the scene's (" + std::to_string(s->n_verts) + ")");
    return RQ_ERR_ARG;
  }
  if (!s->has_tree || !s->d_perm) {
    set_error("scene has no tree to refit");
    return RQ_ERR_STATE;
  }
  if (cudaSetDevice(s->device) != cudaSuccess) {
    set_error("cudaSetDevice");
    return RQ_ERR_CUDA;
  }
  // a topology-keeping refit writes its boxes into the host tree's shape and
  // walks the records level by level: both must be current if rotations
  // changed the tree
  if (mode == RQ_UPDATE_REFIT) {
    if (s->tree_stale && s->tree_from_dyn) {
      const int rc = s->refresh_tree();
      if (rc != RQ_OK) return rc;
    }
    return sync_layout_host(s);
  }
  return RQ_OK;
}

}  // namespace
}  // namespace rq

extern "C" int rq_scene_update_vertices(rq_scene* scene, const float* vertices,
                                        int n_vertices) {
  return rq_scene_update_vertices_ex(scene, vertices, n_vertices, RQ_UPDATE_REFIT);
}

extern "C" int rq_scene_update_vertices_ex(rq_scene* scene, const float* vertices,
                                           int n_vertices, int mode) {
  using namespace rq;
  Scene* s = scene;
  if (!s) {
    set_error("NULL argument");
    return RQ_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->frame_mu);
  int rc = update_begin(s, vertices, n_vertices, mode);
  if (rc != RQ_OK) return rc;
  const size_t nb = 3 * (size_t)n_vertices * sizeof(float);
  std::memcpy(s->verts.data(), vertices, nb);
  s->verts_stale = false;
  const cudaError_t e = cudaMemcpy(s->d_verts, vertices, nb, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    set_error(std::string("update: ") + cudaGetErrorString(e));
    return RQ_ERR_CUDA;
  }
  return update_tree(s, mode);
}

extern "C" int rq_scene_update_vertices_device(rq_scene* scene, const float* d_vertices,
                                               int n_vertices, int mode, void* stream) {
  using namespace rq;
  Scene* s = scene;
  if (!s) {
    set_error("NULL argument");
    return RQ_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->frame_mu);
  int rc = update_begin(s, d_vertices, n_vertices, mode);
  if (rc != RQ_OK) return rc;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t nb = 3 * (size_t)n_vertices * sizeof(float);
  cudaError_t e = cudaMemcpyAsync(s->d_verts, d_vertices, nb, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error(std::string("update: ") + cudaGetErrorString(e));
    return RQ_ERR_CUDA;
  }
  s->verts_stale = true;
  return update_tree(s, mode);
}
