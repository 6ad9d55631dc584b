// Alternative orders of a scene's node records (the "node layout" the
// batched-query autotuner chooses among).  The records themselves (both
// children's boxes, child refs, axis and isLeftCheaper) are unchanged, so a
// traversal visits the same nodes in the same order and returns the same
// bits; only where the records sit in HBM changes, i.e. which records share
// cache lines and DRAM pages with which:
//
//   RQ_LAYOUT_DFS       the builder's depth-first pre-order (a parent's
//                       first child follows it; subtrees are contiguous)
//   RQ_LAYOUT_BFS       breadth-first order from the root (each level of
//                       the tree contiguous, the top levels packed into
//                       the first few cache lines)
//   RQ_LAYOUT_BFS_TOP   the first kTopRecords records in breadth-first
//                       order, then the rest in their depth-first order
//                       (a hot top-of-tree block, subtrees kept together)
//
// The reordered copies are made on the device from the scene's records and
// kept on the scene per layout until its tree changes (generation).
#include <cuda_runtime.h>

#include <algorithm>
#include <deque>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_scene.h"

namespace rq {

constexpr int kTopRecords = 16384;

__global__ void relayout_kernel(const float4* __restrict__ in, float4* __restrict__ out,
                                const int* __restrict__ new_of_old, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = new_of_old[i];
  if (k < 0) return;  // not reachable from the root
  const float4* p = in + 4 * (size_t)i;
  int4 q3 = reinterpret_cast<const int4*>(p)[3];
  if (q3.x >= 0) q3.x = new_of_old[q3.x];
  if (q3.y >= 0) q3.y = new_of_old[q3.y];
  float4* o = out + 4 * (size_t)k;
  o[0] = p[0];
  o[1] = p[1];
  o[2] = p[2];
  reinterpret_cast<int4*>(o)[3] = q3;
}

int Scene::node_layout(int layout, DevScene& S) {
  S = dev();
  if (layout == RQ_LAYOUT_DFS) return RQ_OK;
  if (layout != RQ_LAYOUT_BFS && layout != RQ_LAYOUT_BFS_TOP) {
    set_error("unknown node layout");
    return RQ_ERR_ARG;
  }
  if (!has_tree) {
    set_error("scene has no tree");
    return RQ_ERR_STATE;
  }
  std::lock_guard<std::mutex> g(mu);
  AltLayout& L = alt_layout[layout];
  if (L.nodes && L.generation == generation) {
    S.nodes = L.nodes;
    S.root_ref = L.root;
    return RQ_OK;
  }
  const int n = std::max(n_records, rec_capacity);
  if (root_ref < 0 || n <= 0) return RQ_OK;  // a single leaf: nothing to order
  std::vector<int4> q3(n);
  cudaError_t e = cudaMemcpy2D(q3.data(), sizeof(int4), d_nodes + 3, 4 * sizeof(float4),
                               sizeof(int4), n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    set_error(std::string("layout: ") + cudaGetErrorString(e));
    return RQ_ERR_CUDA;
  }
  // reachable records in breadth-first order
  std::vector<int> bfs;
  bfs.reserve(n);
  std::vector<char> seen(n, 0);
  bfs.push_back(root_ref);
  seen[root_ref] = 1;
  for (size_t h = 0; h < bfs.size(); ++h) {
    const int4 c = q3[bfs[h]];
    for (int ch : {c.x, c.y}) {
      if (ch < 0) continue;
      if (ch >= n || seen[ch]) {
        set_error("layout: malformed node records");
        return RQ_ERR_FORMAT;
      }
      seen[ch] = 1;
      bfs.push_back(ch);
    }
  }
  std::vector<int> new_of_old(n, -1);
  int next = 0;
  if (layout == RQ_LAYOUT_BFS) {
    for (int r : bfs) new_of_old[r] = next++;
  } else {
    const int top = std::min<int>(kTopRecords, (int)bfs.size());
    for (int k = 0; k < top; ++k) new_of_old[bfs[k]] = next++;
    // the rest depth first (near child first, as the builder numbers them)
    std::vector<int> stack;
    stack.push_back(root_ref);
    while (!stack.empty()) {
      const int r = stack.back();
      stack.pop_back();
      if (new_of_old[r] < 0) new_of_old[r] = next++;
      const int4 c = q3[r];
      if (c.y >= 0) stack.push_back(c.y);
      if (c.x >= 0) stack.push_back(c.x);
    }
  }
  const int m = next;
  if (L.nodes && L.capacity < m) {
    cudaFree(L.nodes);
    L.nodes = nullptr;
  }
  int* d_map = nullptr;
  e = cudaSuccess;
  if (!L.nodes) {
    e = cudaMalloc(&L.nodes, (size_t)m * 4 * sizeof(float4));
    L.capacity = m;
  }
  if (e == cudaSuccess) e = cudaMalloc(&d_map, (size_t)n * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(d_map, new_of_old.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    relayout_kernel<<<(n + 255) / 256, 256>>>(d_nodes, L.nodes, d_map, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(d_map);
  if (e != cudaSuccess) {
    set_error(std::string("layout: ") + cudaGetErrorString(e));
    return RQ_ERR_CUDA;
  }
  L.generation = generation;
  L.root = new_of_old[root_ref];
  S.nodes = L.nodes;
  S.root_ref = L.root;
  return RQ_OK;
}

void Scene::free_layouts() {
  for (AltLayout& L : alt_layout) {
    if (L.nodes) cudaFree(L.nodes);
    L = AltLayout();
  }
}

}  // namespace rq
