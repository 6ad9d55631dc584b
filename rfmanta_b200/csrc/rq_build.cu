// GPU binned-SAH builder (rq_scene_build): produces a tree in the reference
// DynBVH form (Model/Groups/DynBVH.h:37-79) - node pairs allocated together,
// leaves as [child, child+children) ranges of object_ids sorted by id - so
// it flows through the same validation and layout path as an imported tree.
//
// Cost model: DynBVH's (Model/Groups/DynBVH.cc:29-30, 2310-2440): split cost
// C_trav + (N_L*A_L + N_R*A_R)/A with C_isec = C_trav = 1, leaf cost N; a
// node becomes a leaf when no split beats the leaf cost (DynBVH::build,
// DynBVH.cc:1804-1857), and a single object is always a leaf.
//
// Algorithm: level-synchronous top-down build, one CTA per node of the
// current level.
//   * n <= 32: the reference's own rule - an exact sweep over the centroid
//     order on every axis (DynBVH::buildEvents, DynBVH.cc:2372-2440), one
//     lane per candidate split;
//   * n > 32: 32 centroid bins per axis accumulated with shared-memory
//     atomics, one warp per axis scanning the bins with shuffles.
// The chosen split partitions the node's index range stably into the other
// half of a ping-pong buffer; leaves write their sorted object ids straight
// into object_ids.  Child pairs are allocated with one atomicAdd.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_internal.h"
#include "rq_scene.h"

namespace rq {

constexpr int kBins = 32;
constexpr int kExactMax = 32;
constexpr int kForceSplit = 255;  // larger nodes are split even when SAH says leaf
constexpr int kBuildThreads = 256;

struct BuildItem {
  int node, begin, end;
};

struct BuildBufs {
  const float* pbox;   // 6 per triangle: min xyz, max xyz
  const float* pcen;   // 3 per triangle: bbox centre
  const int* idx_in;
  int* idx_out;
  int* ids;            // final object_ids
  const BuildItem* items;
  BuildItem* next;
  int* n_next;
  int* node_counter;
  float* nbounds;      // 6 per node
  int* nchild;
  int* nchildren;
  unsigned char* naxis;
};

__device__ __forceinline__ int f2o(float f) {  // order-preserving float -> int
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

__device__ __forceinline__ float area6(const float* b) {
  const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
  return 2.f * (dx * dy + dy * dz + dx * dz);
}

__global__ void prim_bounds_kernel(const float* __restrict__ verts,
                                   const uint32_t* __restrict__ idx, int n,
                                   float* __restrict__ pbox,
                                   float* __restrict__ pcen) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    const float* p = verts + 3 * (size_t)idx[3 * (size_t)t + k];
    for (int c = 0; c < 3; ++c) {
      lo[c] = k == 0 ? p[c] : fminf(lo[c], p[c]);
      hi[c] = k == 0 ? p[c] : fmaxf(hi[c], p[c]);
    }
  }
  for (int c = 0; c < 3; ++c) {
    pbox[6 * (size_t)t + c] = lo[c];
    pbox[6 * (size_t)t + 3 + c] = hi[c];
    pcen[3 * (size_t)t + c] = lo[c] + (hi[c] - lo[c]) * 0.5f;  // BBox::center
  }
}

struct __align__(16) BuildSmem {
  int bcount[3][kBins];
  int bbox[3][kBins][6];  // ordered-int min xyz, max xyz
  float red[kBuildThreads / 32][12];
  float nb[6];   // node bounds
  float cb[6];   // centroid bounds
  float best_cost[3];
  int best_split[3];
  int best_nl[3];
  int decision_axis, decision_split, decision_nl, scan_base[2];
  int wsum[kBuildThreads / 32][2];
  // exact sweep
  float ecen[kExactMax][3];
  float ebox[kExactMax][6];
  int eidx[kExactMax];
  int erank[3][kExactMax];
};

__global__ void __launch_bounds__(kBuildThreads) build_level_kernel(BuildBufs B) {
  __shared__ BuildSmem s;
  const BuildItem it = B.items[blockIdx.x];
  const int b = it.begin, e = it.end, n = e - b;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  // ---- node bounds and centroid bounds --------------------------------
  float v[12];
  for (int c = 0; c < 3; ++c) {
    v[c] = INFINITY;
    v[3 + c] = -INFINITY;
    v[6 + c] = INFINITY;
    v[9 + c] = -INFINITY;
  }
  for (int i = b + tid; i < e; i += blockDim.x) {
    const int p = B.idx_in[i];
    for (int c = 0; c < 3; ++c) {
      v[c] = fminf(v[c], B.pbox[6 * (size_t)p + c]);
      v[3 + c] = fmaxf(v[3 + c], B.pbox[6 * (size_t)p + 3 + c]);
      const float cc = B.pcen[3 * (size_t)p + c];
      v[6 + c] = fminf(v[6 + c], cc);
      v[9 + c] = fmaxf(v[9 + c], cc);
    }
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int c = 0; c < 3; ++c) {
      v[c] = fminf(v[c], __shfl_xor_sync(0xffffffffu, v[c], o));
      v[3 + c] = fmaxf(v[3 + c], __shfl_xor_sync(0xffffffffu, v[3 + c], o));
      v[6 + c] = fminf(v[6 + c], __shfl_xor_sync(0xffffffffu, v[6 + c], o));
      v[9 + c] = fmaxf(v[9 + c], __shfl_xor_sync(0xffffffffu, v[9 + c], o));
    }
  if (lane == 0)
    for (int k = 0; k < 12; ++k) s.red[warp][k] = v[k];
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < (int)(blockDim.x / 32); ++w)
      for (int c = 0; c < 3; ++c) {
        s.red[0][c] = fminf(s.red[0][c], s.red[w][c]);
        s.red[0][3 + c] = fmaxf(s.red[0][3 + c], s.red[w][3 + c]);
        s.red[0][6 + c] = fminf(s.red[0][6 + c], s.red[w][6 + c]);
        s.red[0][9 + c] = fmaxf(s.red[0][9 + c], s.red[w][9 + c]);
      }
    for (int k = 0; k < 6; ++k) {
      s.nb[k] = s.red[0][k];
      s.cb[k] = s.red[0][6 + k];
      B.nbounds[6 * (size_t)it.node + k] = s.red[0][k];
    }
    s.decision_axis = -1;
    for (int a = 0; a < 3; ++a) s.best_cost[a] = INFINITY;
  }
  __syncthreads();
  const float parea = area6(s.nb);

  if (n > 1 && n <= kExactMax) {
    // ---- exact sweep (DynBVH::buildEvents) ------------------------------
    if (tid < n) {
      const int p = B.idx_in[b + tid];
      s.eidx[tid] = p;
      for (int c = 0; c < 3; ++c) s.ecen[tid][c] = B.pcen[3 * (size_t)p + c];
      for (int k = 0; k < 6; ++k) s.ebox[tid][k] = B.pbox[6 * (size_t)p + k];
    }
    __syncthreads();
    if (warp < 3) {
      const int a = warp;
      if (lane < n) {
        const float ci = s.ecen[lane][a];
        int r = 0;
        for (int j = 0; j < n; ++j) {
          const float cj = s.ecen[j][a];
          r += (cj < ci || (cj == ci && j < lane)) ? 1 : 0;
        }
        s.erank[a][lane] = r;
      }
      __syncwarp();
      // candidate: left = ranks [0, r), r = lane + 1 in [1, n-1]
      float cost = INFINITY;
      const int r = lane + 1;
      if (r < n) {
        float L[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        float R[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (int j = 0; j < n; ++j) {
          float* D = s.erank[a][j] < r ? L : R;
          for (int c = 0; c < 3; ++c) {
            D[c] = fminf(D[c], s.ebox[j][c]);
            D[3 + c] = fmaxf(D[3 + c], s.ebox[j][3 + c]);
          }
        }
        cost = 1.f + ((float)r * area6(L) + (float)(n - r) * area6(R)) / parea;
      }
      float bc = cost;
      int bl = lane;
      for (int o = 16; o > 0; o >>= 1) {
        const float oc = __shfl_xor_sync(0xffffffffu, bc, o);
        const int ol = __shfl_xor_sync(0xffffffffu, bl, o);
        if (oc < bc || (oc == bc && ol < bl)) {
          bc = oc;
          bl = ol;
        }
      }
      if (lane == 0) {
        s.best_cost[a] = bc;
        s.best_split[a] = bl + 1;
        s.best_nl[a] = bl + 1;
      }
    }
    __syncthreads();
  } else if (n > kExactMax) {
    // ---- binned SAH ------------------------------------------------------
    for (int k = tid; k < 3 * kBins; k += blockDim.x) {
      const int a = k / kBins, bin = k % kBins;
      s.bcount[a][bin] = 0;
      for (int c = 0; c < 3; ++c) {
        s.bbox[a][bin][c] = f2o(INFINITY);
        s.bbox[a][bin][3 + c] = f2o(-INFINITY);
      }
    }
    __syncthreads();
    float scale[3];
    for (int a = 0; a < 3; ++a) {
      const float ext = s.cb[3 + a] - s.cb[a];
      scale[a] = ext > 0.f ? (float)kBins / ext : 0.f;
    }
    for (int i = b + tid; i < e; i += blockDim.x) {
      const int p = B.idx_in[i];
      float pb[6];
      for (int k = 0; k < 6; ++k) pb[k] = B.pbox[6 * (size_t)p + k];
      for (int a = 0; a < 3; ++a) {
        if (scale[a] == 0.f) continue;
        const int bin = min(kBins - 1, (int)((B.pcen[3 * (size_t)p + a] - s.cb[a]) * scale[a]));
        atomicAdd(&s.bcount[a][bin], 1);
        for (int c = 0; c < 3; ++c) {
          atomicMin(&s.bbox[a][bin][c], f2o(pb[c]));
          atomicMax(&s.bbox[a][bin][3 + c], f2o(pb[3 + c]));
        }
      }
    }
    __syncthreads();
    if (warp < 3) {
      const int a = warp;
      float cost = INFINITY;
      int nl = 0;
      if (scale[a] != 0.f) {
        const int cnt = s.bcount[a][lane];
        float bx[6];
        for (int k = 0; k < 6; ++k) bx[k] = o2f(s.bbox[a][lane][k]);
        // inclusive prefix (left) and suffix (right) scans over the 32 bins
        int lc = cnt, rc = cnt;
        float lb[6], rb[6];
        for (int k = 0; k < 6; ++k) lb[k] = rb[k] = bx[k];
        for (int o = 1; o < 32; o <<= 1) {
          const int tl = __shfl_up_sync(0xffffffffu, lc, o);
          const int tr = __shfl_down_sync(0xffffffffu, rc, o);
          float ul[6], dr[6];
          for (int k = 0; k < 6; ++k) {
            ul[k] = __shfl_up_sync(0xffffffffu, lb[k], o);
            dr[k] = __shfl_down_sync(0xffffffffu, rb[k], o);
          }
          if (lane >= o) {
            lc += tl;
            for (int c = 0; c < 3; ++c) {
              lb[c] = fminf(lb[c], ul[c]);
              lb[3 + c] = fmaxf(lb[3 + c], ul[3 + c]);
            }
          }
          if (lane + o < 32) {
            rc += tr;
            for (int c = 0; c < 3; ++c) {
              rb[c] = fminf(rb[c], dr[c]);
              rb[3 + c] = fmaxf(rb[3 + c], dr[3 + c]);
            }
          }
        }
        // split after bin `lane`: left = bins [0, lane], right = (lane, 31]
        const int rcn = __shfl_down_sync(0xffffffffu, rc, 1);
        float rbn[6];
        for (int k = 0; k < 6; ++k) rbn[k] = __shfl_down_sync(0xffffffffu, rb[k], 1);
        if (lane < 31 && lc > 0 && rcn > 0) {
          cost = 1.f + ((float)lc * area6(lb) + (float)rcn * area6(rbn)) / parea;
          nl = lc;
        }
      }
      float bc = cost;
      int bl = lane, bn = nl;
      for (int o = 16; o > 0; o >>= 1) {
        const float oc = __shfl_xor_sync(0xffffffffu, bc, o);
        const int ol = __shfl_xor_sync(0xffffffffu, bl, o);
        const int on = __shfl_xor_sync(0xffffffffu, bn, o);
        if (oc < bc || (oc == bc && ol < bl)) {
          bc = oc;
          bl = ol;
          bn = on;
        }
      }
      if (lane == 0) {
        s.best_cost[a] = bc;
        s.best_split[a] = bl;
        s.best_nl[a] = bn;
      }
    }
    __syncthreads();
  }

  // ---- decision ------------------------------------------------------------
  if (tid == 0) {
    int ba = -1;
    float bc = INFINITY;
    for (int a = 0; a < 3; ++a)
      if (s.best_cost[a] < bc) {
        bc = s.best_cost[a];
        ba = a;
      }
    const bool split = n > 1 && ba >= 0 && (bc < (float)n || n > kForceSplit);
    s.decision_axis = split ? ba : -1;
    if (split) {
      s.decision_split = s.best_split[ba];
      s.decision_nl = s.best_nl[ba];
    } else if (n > kForceSplit) {
      // no usable plane at all (identical centroids): object median
      s.decision_axis = 0;
      s.decision_split = -1;
      s.decision_nl = n / 2;
    }
  }
  __syncthreads();
  const int axis = s.decision_axis;
  if (axis < 0) {
    // leaf: object ids in increasing order (DynBVH.cc:1837 std::sort)
    if (tid == 0) {
      B.nchild[it.node] = b;
      B.nchildren[it.node] = n;
      B.naxis[it.node] = 0;
    }
    if (n <= kBuildThreads) {
      const int p = tid < n ? B.idx_in[b + tid] : 0x7fffffff;
      int r = 0;
      if (tid < n)
        for (int j = 0; j < n; ++j) r += B.idx_in[b + j] < p ? 1 : 0;
      if (tid < n) B.ids[b + r] = p;
    } else {
      for (int i = b + tid; i < e; i += blockDim.x) B.ids[i] = B.idx_in[i];
    }
    return;
  }
  // ---- stable partition into idx_out -------------------------------------
  const int nl = s.decision_nl;
  const bool exact = n <= kExactMax;
  const bool median = s.decision_split < 0;
  float scale_a = 0.f;
  if (!exact && !median) scale_a = (float)kBins / (s.cb[3 + axis] - s.cb[axis]);
  if (tid == 0) {
    s.scan_base[0] = 0;
    s.scan_base[1] = 0;
  }
  __syncthreads();
  for (int base = b; base < e; base += blockDim.x) {
    const int i = base + tid;
    int p = 0;
    bool left = false;
    if (i < e) {
      p = B.idx_in[i];
      if (exact)
        left = s.erank[axis][i - b] < s.decision_split;
      else if (median)
        left = (i - b) < nl;
      else
        left = min(kBins - 1, (int)((B.pcen[3 * (size_t)p + axis] - s.cb[axis]) * scale_a)) <=
               s.decision_split;
    }
    const unsigned ml = __ballot_sync(0xffffffffu, i < e && left);
    const unsigned mr = __ballot_sync(0xffffffffu, i < e && !left);
    if (lane == 0) {
      s.wsum[warp][0] = __popc(ml);
      s.wsum[warp][1] = __popc(mr);
    }
    __syncthreads();
    int offl = s.scan_base[0], offr = s.scan_base[1];
    for (int w = 0; w < warp; ++w) {
      offl += s.wsum[w][0];
      offr += s.wsum[w][1];
    }
    const unsigned lt = (1u << lane) - 1u;
    if (i < e) {
      if (left)
        B.idx_out[b + offl + __popc(ml & lt)] = p;
      else
        B.idx_out[b + nl + offr + __popc(mr & lt)] = p;
    }
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
        s.scan_base[0] += s.wsum[w][0];
        s.scan_base[1] += s.wsum[w][1];
      }
    __syncthreads();
  }
  if (tid == 0) {
    const int c = atomicAdd(B.node_counter, 2);
    B.nchild[it.node] = c;
    B.nchildren[it.node] = 0;
    B.naxis[it.node] = (unsigned char)axis;
    const int q = atomicAdd(B.n_next, 2);
    B.next[q] = BuildItem{c, b, b + nl};
    B.next[q + 1] = BuildItem{c + 1, b + nl, e};
  }
}

template <class T>
static cudaError_t dalloc(T** p, size_t n) {
  return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T));
}

// Builds the tree into `out` (host, reference field-wise form).
int gpu_build(Scene* s, HostTree& out, double* seconds) {
  const int n = s->n_tris;
  float *pbox = nullptr, *pcen = nullptr, *nb = nullptr;
  int *ia = nullptr, *ib = nullptr, *ids = nullptr, *nchild = nullptr, *nchildren = nullptr;
  int *counters = nullptr;
  unsigned char* naxis = nullptr;
  BuildItem *items_a = nullptr, *items_b = nullptr;
  const size_t max_nodes = 2 * (size_t)n;
  cudaError_t e = cudaSuccess;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto cleanup = [&]() {
    cudaFree(pbox); cudaFree(pcen); cudaFree(nb); cudaFree(ia); cudaFree(ib); cudaFree(ids);
    cudaFree(nchild); cudaFree(nchildren); cudaFree(counters); cudaFree(naxis);
    cudaFree(items_a); cudaFree(items_b);
    cudaEventDestroy(t0); cudaEventDestroy(t1);
  };
#define BCHK(x)                                                         \
  do {                                                                  \
    e = (x);                                                            \
    if (e != cudaSuccess) {                                             \
      set_error(std::string("builder: ") + #x + ": " + cudaGetErrorString(e)); \
      cleanup();                                                        \
      return e == cudaErrorMemoryAllocation ? RQ_ERR_OOM : RQ_ERR_CUDA; \
    }                                                                   \
  } while (0)
  BCHK(dalloc(&pbox, 6 * (size_t)n));
  BCHK(dalloc(&pcen, 3 * (size_t)n));
  BCHK(dalloc(&nb, 6 * max_nodes));
  BCHK(dalloc(&ia, n));
  BCHK(dalloc(&ib, n));
  BCHK(dalloc(&ids, n));
  BCHK(dalloc(&nchild, max_nodes));
  BCHK(dalloc(&nchildren, max_nodes));
  BCHK(dalloc(&naxis, max_nodes));
  BCHK(dalloc(&counters, 4));
  BCHK(dalloc(&items_a, n));
  BCHK(dalloc(&items_b, n));
  BCHK(cudaEventRecord(t0, 0));
  prim_bounds_kernel<<<(n + 255) / 256, 256>>>(s->d_verts, s->d_idx, n, pbox, pcen);
  BCHK(cudaGetLastError());
  {
    std::vector<int> iota(n);
    for (int i = 0; i < n; ++i) iota[i] = i;
    BCHK(cudaMemcpy(ia, iota.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
  }
  const int init[4] = {1, 0, 0, 0};
  BCHK(cudaMemcpy(counters, init, sizeof(init), cudaMemcpyHostToDevice));
  const BuildItem root{0, 0, n};
  BCHK(cudaMemcpy(items_a, &root, sizeof(root), cudaMemcpyHostToDevice));
  int n_items = 1;
  int* idx_in = ia;
  int* idx_out = ib;
  BuildItem* cur = items_a;
  BuildItem* nxt = items_b;
  int levels = 0;
  while (n_items > 0) {
    BCHK(cudaMemsetAsync(counters + 1, 0, sizeof(int), 0));
    BuildBufs B{pbox, pcen, idx_in, idx_out, ids, cur, nxt, counters + 1, counters,
                nb, nchild, nchildren, naxis};
    build_level_kernel<<<n_items, kBuildThreads>>>(B);
    BCHK(cudaGetLastError());
    BCHK(cudaMemcpy(&n_items, counters + 1, sizeof(int), cudaMemcpyDeviceToHost));
    std::swap(idx_in, idx_out);
    std::swap(cur, nxt);
    if (++levels > 4096) {
      set_error("builder: too many levels");
      cleanup();
      return RQ_ERR_CAPACITY;
    }
  }
  BCHK(cudaEventRecord(t1, 0));
  BCHK(cudaEventSynchronize(t1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  if (seconds) *seconds = ms * 1e-3;
  int nn = 0;
  BCHK(cudaMemcpy(&nn, counters, sizeof(int), cudaMemcpyDeviceToHost));
  out.bounds.resize(6 * (size_t)nn);
  out.child.resize(nn);
  out.children.resize(nn);
  out.axis.resize(nn);
  out.left_cheaper.assign(nn, 1);
  out.ids.resize(n);
  BCHK(cudaMemcpy(out.bounds.data(), nb, 24 * (size_t)nn, cudaMemcpyDeviceToHost));
  BCHK(cudaMemcpy(out.child.data(), nchild, 4 * (size_t)nn, cudaMemcpyDeviceToHost));
  BCHK(cudaMemcpy(out.children.data(), nchildren, 4 * (size_t)nn, cudaMemcpyDeviceToHost));
  BCHK(cudaMemcpy(out.axis.data(), naxis, (size_t)nn, cudaMemcpyDeviceToHost));
  BCHK(cudaMemcpy(out.ids.data(), ids, 4 * (size_t)n, cudaMemcpyDeviceToHost));
#undef BCHK
  cleanup();
  // Any-hit child order: the child with the smaller SAH subtree cost first
  // (the reference ranks children by its RTSAH cost, DynBVH.cc:1594-1678;
  // the order only affects speed, never which rays are occluded).
  std::vector<float> cost(nn, 0.f);
  std::vector<int> order;
  order.reserve(nn);
  std::vector<int> st(1, 0);
  while (!st.empty()) {
    const int k = st.back();
    st.pop_back();
    order.push_back(k);
    if (out.children[k] == 0) {
      st.push_back(out.child[k]);
      st.push_back(out.child[k] + 1);
    }
  }
  auto area = [&](int k) {
    const float* b = &out.bounds[6 * (size_t)k];
    const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return 2 * (dx * dy + dy * dz + dx * dz);
  };
  for (size_t i = order.size(); i-- > 0;) {
    const int k = order[i];
    if (out.children[k] != 0) {
      cost[k] = (float)out.children[k];
    } else {
      const int L = out.child[k], R = L + 1;
      const float a = area(k);
      cost[k] = 1.f + (area(L) * cost[L] + area(R) * cost[R]) / a;
      out.left_cheaper[k] = area(L) * cost[L] <= area(R) * cost[R] ? 1 : 0;
    }
  }
  return RQ_OK;
}

}  // namespace rq

extern "C" int rq_scene_build(rq_scene* scene, int bins) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s) {
    rq::set_error("NULL scene");
    return RQ_ERR_ARG;
  }
  if (bins != 0 && bins != rq::kBins) {
    rq::set_error("this builder uses 32 bins (pass 0 or 32)");
    return RQ_ERR_ARG;
  }
  if (cudaSetDevice(s->device) != cudaSuccess) {
    rq::set_error("cudaSetDevice failed");
    return RQ_ERR_CUDA;
  }
  rq::HostTree t;
  double secs = 0;
  int rc = rq::gpu_build(s, t, &secs);
  if (rc != RQ_OK) return rc;
  s->last_build_seconds = secs;
  return s->set_tree(t);
}
