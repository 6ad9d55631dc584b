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
// current level (nodes of more than kBigNode primitives in a level of few
// nodes: one CTA per slice of the node, see below).
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

// ---- large nodes: many CTAs per node --------------------------------------
//
// The top levels hold few nodes with many primitives each; one CTA per node
// would leave most SMs idle.  Nodes with more than kBigNode primitives are
// cut into slices of kSlice primitives and processed by one CTA per slice:
// bounds (global atomic min/max), binning (shared-memory bins merged into
// the node's global bins), one CTA per node for the SAH decision (the same
// scans and rules as build_level_kernel), then a stable partition: per-slice
// left counts, their prefix per node, and a scatter that keeps each slice's
// order.  Bin counts and min/max bounds do not depend on the order of the
// atomics and the partition is stable, so a node gets the same split and the
// same child ranges as the one-CTA path would give it.
constexpr int kBigNode = 1 << 16;
constexpr int kSlice = 8192;

struct BigAcc {
  int nb[6];  // ordered-int node bounds: min xyz, max xyz
  int cb[6];  // ordered-int centroid bounds
  int bcount[3][kBins];
  int bbox[3][kBins][6];
  // decision (written by big_decide_kernel)
  int axis, split, nl, median;
  float cb_f[6];
};

struct BigSlice {
  int node;  // index into the level's big nodes
  int begin, end;
  int offl, offr;  // left / right elements of earlier slices of the node
  int nleft;
};

__global__ void big_init_kernel(BigAcc* acc, int n_big) {
  const int k = blockIdx.x;
  if (k >= n_big) return;
  BigAcc& A = acc[k];
  for (int i = threadIdx.x; i < 3 * kBins; i += blockDim.x) {
    const int a = i / kBins, bin = i % kBins;
    A.bcount[a][bin] = 0;
    for (int c = 0; c < 3; ++c) {
      A.bbox[a][bin][c] = f2o(INFINITY);
      A.bbox[a][bin][3 + c] = f2o(-INFINITY);
    }
  }
  if (threadIdx.x < 3) {
    A.nb[threadIdx.x] = f2o(INFINITY);
    A.nb[3 + threadIdx.x] = f2o(-INFINITY);
    A.cb[threadIdx.x] = f2o(INFINITY);
    A.cb[3 + threadIdx.x] = f2o(-INFINITY);
  }
}

__global__ void __launch_bounds__(kBuildThreads)
    big_bounds_kernel(BuildBufs B, const BigSlice* slices, BigAcc* acc) {
  __shared__ float red[kBuildThreads / 32][12];
  const BigSlice sl = slices[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float v[12];
  for (int c = 0; c < 3; ++c) {
    v[c] = INFINITY;
    v[3 + c] = -INFINITY;
    v[6 + c] = INFINITY;
    v[9 + c] = -INFINITY;
  }
  for (int i = sl.begin + tid; i < sl.end; i += blockDim.x) {
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
    for (int k = 0; k < 12; ++k) red[warp][k] = v[k];
  __syncthreads();
  if (tid < 12) {
    float x = red[0][tid];
    for (int w = 1; w < (int)(blockDim.x / 32); ++w) {
      const bool mn = (tid % 6) < 3;
      x = mn ? fminf(x, red[w][tid]) : fmaxf(x, red[w][tid]);
    }
    BigAcc& A = acc[sl.node];
    int* dst = tid < 6 ? &A.nb[tid] : &A.cb[tid - 6];
    if ((tid % 6) < 3)
      atomicMin(dst, f2o(x));
    else
      atomicMax(dst, f2o(x));
  }
}

__global__ void __launch_bounds__(kBuildThreads)
    big_bin_kernel(BuildBufs B, const BigSlice* slices, BigAcc* acc) {
  __shared__ int bcount[3][kBins];
  __shared__ int bbox[3][kBins][6];
  const BigSlice sl = slices[blockIdx.x];
  BigAcc& A = acc[sl.node];
  const int tid = threadIdx.x;
  for (int k = tid; k < 3 * kBins; k += blockDim.x) {
    const int a = k / kBins, bin = k % kBins;
    bcount[a][bin] = 0;
    for (int c = 0; c < 3; ++c) {
      bbox[a][bin][c] = f2o(INFINITY);
      bbox[a][bin][3 + c] = f2o(-INFINITY);
    }
  }
  float cb[6], scale[3];
  for (int k = 0; k < 6; ++k) cb[k] = o2f(A.cb[k]);
  for (int a = 0; a < 3; ++a) {
    const float ext = cb[3 + a] - cb[a];
    scale[a] = ext > 0.f ? (float)kBins / ext : 0.f;
  }
  __syncthreads();
  for (int i = sl.begin + tid; i < sl.end; i += blockDim.x) {
    const int p = B.idx_in[i];
    float pb[6];
    for (int k = 0; k < 6; ++k) pb[k] = B.pbox[6 * (size_t)p + k];
    for (int a = 0; a < 3; ++a) {
      if (scale[a] == 0.f) continue;
      const int bin = min(kBins - 1, (int)((B.pcen[3 * (size_t)p + a] - cb[a]) * scale[a]));
      atomicAdd(&bcount[a][bin], 1);
      for (int c = 0; c < 3; ++c) {
        atomicMin(&bbox[a][bin][c], f2o(pb[c]));
        atomicMax(&bbox[a][bin][3 + c], f2o(pb[3 + c]));
      }
    }
  }
  __syncthreads();
  for (int k = tid; k < 3 * kBins; k += blockDim.x) {
    const int a = k / kBins, bin = k % kBins;
    if (bcount[a][bin] == 0) continue;
    atomicAdd(&A.bcount[a][bin], bcount[a][bin]);
    for (int c = 0; c < 3; ++c) {
      atomicMin(&A.bbox[a][bin][c], bbox[a][bin][c]);
      atomicMax(&A.bbox[a][bin][3 + c], bbox[a][bin][3 + c]);
    }
  }
}

// One CTA (3 warps used) per large node: the binned SAH sweep and the split
// decision of build_level_kernel, from the node's merged bins.
__global__ void big_decide_kernel(BuildBufs B, const BuildItem* items, BigAcc* acc) {
  __shared__ float best_cost[3];
  __shared__ int best_split[3], best_nl[3];
  const BuildItem it = items[blockIdx.x];
  BigAcc& A = acc[blockIdx.x];
  const int n = it.end - it.begin;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float nb[6], cb[6];
  for (int k = 0; k < 6; ++k) {
    nb[k] = o2f(A.nb[k]);
    cb[k] = o2f(A.cb[k]);
  }
  const float parea = area6(nb);
  if (warp < 3) {
    const int a = warp;
    const float ext = cb[3 + a] - cb[a];
    const bool usable = ext > 0.f;
    float cost = INFINITY;
    int nl = 0;
    if (usable) {
      const int cnt = A.bcount[a][lane];
      float bx[6];
      for (int k = 0; k < 6; ++k) bx[k] = o2f(A.bbox[a][lane][k]);
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
      best_cost[a] = usable ? bc : INFINITY;
      best_split[a] = bl;
      best_nl[a] = bn;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int ba = -1;
    float bc = INFINITY;
    for (int a = 0; a < 3; ++a)
      if (best_cost[a] < bc) {
        bc = best_cost[a];
        ba = a;
      }
    // n > kForceSplit always holds here: the node is split, by SAH when a
    // plane exists, else at the object median
    if (ba >= 0) {
      A.axis = ba;
      A.split = best_split[ba];
      A.nl = best_nl[ba];
      A.median = 0;
    } else {
      A.axis = 0;
      A.split = -1;
      A.nl = n / 2;
      A.median = 1;
    }
    for (int k = 0; k < 6; ++k) {
      A.cb_f[k] = cb[k];
      B.nbounds[6 * (size_t)it.node + k] = nb[k];
    }
  }
}

__device__ __forceinline__ bool big_left(const BuildBufs& B, const BigAcc& A, int b, int i,
                                         int p, float scale_a) {
  if (A.median) return (i - b) < A.nl;
  return min(kBins - 1, (int)((B.pcen[3 * (size_t)p + A.axis] - A.cb_f[A.axis]) * scale_a)) <=
         A.split;
}

__global__ void __launch_bounds__(kBuildThreads)
    big_count_kernel(BuildBufs B, const BuildItem* items, BigSlice* slices, const BigAcc* acc) {
  __shared__ int wsum[kBuildThreads / 32];
  BigSlice& sl = slices[blockIdx.x];
  const BigAcc& A = acc[sl.node];
  const int b = items[sl.node].begin;
  const float scale_a = A.median ? 0.f : (float)kBins / (A.cb_f[3 + A.axis] - A.cb_f[A.axis]);
  int c = 0;
  for (int i = sl.begin + threadIdx.x; i < sl.end; i += blockDim.x)
    c += big_left(B, A, b, i, B.idx_in[i], scale_a) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += wsum[w];
    sl.nleft = t;
  }
}

// Per large node (one thread each): offsets of its slices, then the child
// pair and the next level's two items.
__global__ void big_offsets_kernel(BuildBufs B, const BuildItem* items, BigSlice* slices,
                                   int n_slices, const BigAcc* acc, int n_big) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_big) return;
  int offl = 0, offr = 0;
  for (int j = 0; j < n_slices; ++j) {
    if (slices[j].node != k) continue;
    slices[j].offl = offl;
    slices[j].offr = offr;
    offl += slices[j].nleft;
    offr += (slices[j].end - slices[j].begin) - slices[j].nleft;
  }
  const BuildItem it = items[k];
  const int nl = acc[k].nl;
  const int c = atomicAdd(B.node_counter, 2);
  B.nchild[it.node] = c;
  B.nchildren[it.node] = 0;
  B.naxis[it.node] = (unsigned char)acc[k].axis;
  const int q = atomicAdd(B.n_next, 2);
  B.next[q] = BuildItem{c, it.begin, it.begin + nl};
  B.next[q + 1] = BuildItem{c + 1, it.begin + nl, it.end};
}

__global__ void __launch_bounds__(kBuildThreads)
    big_scatter_kernel(BuildBufs B, const BuildItem* items, const BigSlice* slices,
                       const BigAcc* acc) {
  __shared__ int wsum[kBuildThreads / 32][2];
  __shared__ int base[2];
  const BigSlice sl = slices[blockIdx.x];
  const BigAcc& A = acc[sl.node];
  const int b = items[sl.node].begin, e = items[sl.node].end;
  const int nl = A.nl;
  const float scale_a = A.median ? 0.f : (float)kBins / (A.cb_f[3 + A.axis] - A.cb_f[A.axis]);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    base[0] = sl.offl;
    base[1] = sl.offr;
  }
  __syncthreads();
  for (int start = sl.begin; start < sl.end; start += blockDim.x) {
    const int i = start + tid;
    int p = 0;
    bool left = false;
    if (i < sl.end) {
      p = B.idx_in[i];
      left = big_left(B, A, b, i, p, scale_a);
    }
    const unsigned ml = __ballot_sync(0xffffffffu, i < sl.end && left);
    const unsigned mr = __ballot_sync(0xffffffffu, i < sl.end && !left);
    if (lane == 0) {
      wsum[warp][0] = __popc(ml);
      wsum[warp][1] = __popc(mr);
    }
    __syncthreads();
    int offl = base[0], offr = base[1];
    for (int w = 0; w < warp; ++w) {
      offl += wsum[w][0];
      offr += wsum[w][1];
    }
    const unsigned lt = (1u << lane) - 1u;
    if (i < sl.end) {
      // the node's left count nl comes from the same bin rule, so every
      // destination lies in [b, e); the guard keeps a write inside the node
      // even if it did not
      const int d = left ? b + offl + __popc(ml & lt) : b + nl + offr + __popc(mr & lt);
      if (d >= b && d < e) B.idx_out[d] = p;
    }
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
        base[0] += wsum[w][0];
        base[1] += wsum[w][1];
      }
    __syncthreads();
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
  // large-node path: per-node accumulators, slice table, item lists
  const int max_big = n / kBigNode + 1;
  const int max_slices = n / kSlice + max_big + 1;
  constexpr int kHostItems = 512;  // levels this small are split on the host
  BigAcc* acc = nullptr;
  BigSlice* slices = nullptr;
  BuildItem *big_items = nullptr, *small_items = nullptr;
  const size_t max_nodes = 2 * (size_t)n;
  cudaError_t e = cudaSuccess;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto cleanup = [&]() {
    cudaFree(pbox); cudaFree(pcen); cudaFree(nb); cudaFree(ia); cudaFree(ib); cudaFree(ids);
    cudaFree(nchild); cudaFree(nchildren); cudaFree(counters); cudaFree(naxis);
    cudaFree(items_a); cudaFree(items_b);
    cudaFree(acc); cudaFree(slices); cudaFree(big_items); cudaFree(small_items);
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
  BCHK(dalloc(&acc, max_big));
  BCHK(dalloc(&slices, max_slices));
  BCHK(dalloc(&big_items, max_big));
  BCHK(dalloc(&small_items, kHostItems));
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
  std::vector<BuildItem> h_items, h_big, h_small;
  std::vector<BigSlice> h_slices;
  while (n_items > 0) {
    BCHK(cudaMemsetAsync(counters + 1, 0, sizeof(int), 0));
    BuildBufs B{pbox, pcen, idx_in, idx_out, ids, cur, nxt, counters + 1, counters,
                nb, nchild, nchildren, naxis};
    // a level of few nodes: nodes above kBigNode primitives go to the
    // many-CTA path, the rest to build_level_kernel
    h_big.clear();
    h_small.clear();
    if (n_items <= kHostItems) {
      h_items.resize(n_items);
      BCHK(cudaMemcpy(h_items.data(), cur, sizeof(BuildItem) * n_items, cudaMemcpyDeviceToHost));
      for (const BuildItem& it : h_items)
        (it.end - it.begin > kBigNode ? h_big : h_small).push_back(it);
    }
    if (!h_big.empty()) {
      h_slices.clear();
      for (int k = 0; k < (int)h_big.size(); ++k)
        for (int b0 = h_big[k].begin; b0 < h_big[k].end; b0 += kSlice)
          h_slices.push_back(BigSlice{k, b0, std::min(b0 + kSlice, h_big[k].end), 0, 0, 0});
      const int nbig = (int)h_big.size(), nsl = (int)h_slices.size();
      BCHK(cudaMemcpy(big_items, h_big.data(), sizeof(BuildItem) * nbig, cudaMemcpyHostToDevice));
      BCHK(cudaMemcpy(slices, h_slices.data(), sizeof(BigSlice) * nsl, cudaMemcpyHostToDevice));
      big_init_kernel<<<nbig, 128>>>(acc, nbig);
      big_bounds_kernel<<<nsl, kBuildThreads>>>(B, slices, acc);
      big_bin_kernel<<<nsl, kBuildThreads>>>(B, slices, acc);
      big_decide_kernel<<<nbig, 96>>>(B, big_items, acc);
      big_count_kernel<<<nsl, kBuildThreads>>>(B, big_items, slices, acc);
      big_offsets_kernel<<<(nbig + 31) / 32, 32>>>(B, big_items, slices, nsl, acc, nbig);
      big_scatter_kernel<<<nsl, kBuildThreads>>>(B, big_items, slices, acc);
      BCHK(cudaGetLastError());
      if (!h_small.empty()) {
        BCHK(cudaMemcpy(small_items, h_small.data(), sizeof(BuildItem) * h_small.size(),
                        cudaMemcpyHostToDevice));
        BuildBufs Bs = B;
        Bs.items = small_items;
        build_level_kernel<<<(int)h_small.size(), kBuildThreads>>>(Bs);
      }
    } else {
      build_level_kernel<<<n_items, kBuildThreads>>>(B);
    }
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
  rq::park_channels(s);  // the build's allocations would wait for a running channel
  rq::HostTree t;
  double secs = 0;
  int rc = rq::gpu_build(s, t, &secs);
  if (rc != RQ_OK) return rc;
  s->last_build_seconds = secs;
  return s->set_tree(t);
}
