// The reference's DynBVH::update for an animated mesh as it ships
// (Model/Groups/DynBVH.cc:1574-1581 with TREE_ROT 1, DynBVH.h:377): after
// the vertices move, every node box is recomputed bottom up
// (updateBounds, 2068-2123) and, at every internal node, rotateNode
// (3051-3348, Kopta et al. 2012) first re-splits leaf children holding more
// than one object with the approximate binned build (build 1807-1857,
// partitionApproxSAH 2125-2275, partition2Objs 2277-2307, partitionObjects
// 1369-1396), then applies the best of six child/grandchild swaps by SAH
// cost, updates the per-node costs and re-guesses the split axes.  The
// result is the reference's tree, field for field, and the per-node costs
// and next free node the next frame starts from.
//
// The reference walks the tree once, recursively, in post order.  Here:
//   1. object boxes and centroids, one thread per triangle;
//   2. leaf boxes (and each node's parent), one thread per record child;
//   3. leaf re-splits, one thread per leaf, into per-leaf scratch.  A leaf is
//      re-split by its parent's rotateNode, before anything else touches it,
//      and the split depends only on the leaf's objects, so all splits can
//      run first.  Only where their nodes go depends on the order: the
//      reference hands out node pairs from one counter in post order of the
//      parents (left child before right), so the split sizes are scanned in
//      that order (post(r) = pre(r) - depth(r) + size(r) - 1 for a record in
//      pre-order) and every split is copied to its own offset;
//   4. rotations bottom up: one thread per original leaf climbs towards the
//      root; the second thread to arrive at a node handles it.  A rotation
//      at a node reads and writes only its children and grandchildren, all
//      inside its finished subtree, so the order across subtrees is free;
//   5. the traversal records, leaf object order and triangle records are
//      laid out again from the rotated tree, one tree level per launch.
// Float arithmetic follows the reference's operation order with explicitly
// rounded operations; Min/Max are its ternaries (Core/Math/MinMax.h:83-91),
// boxes start from [FLT_MAX, -FLT_MAX] (BBox::reset), BBox::computeArea is
// float arithmetic widened to double, Vector::indexOfMaxComponent gives ties
// to the later component (Core/Geometry/Vector.h:382-394), and int(float)
// is x86's truncation (NaN and out-of-range values give INT_MIN).
// isLargeSubtree and subtree_size only steer the reference's multi-threaded
// update and are not kept; the result is that of DynBVH::update(0, 1).
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_internal.h"
#include "rq_scene.h"

namespace rq {

// Results of an update on the device, read back once at its end.
struct UpdState {
  int next_free;
  int error;  // 1: node capacity, 2: deeper than the traversal stack, 3: record capacity
  int n_records;
  int depth;
  float root[6];
};

// Device state of the rotating update: the reference's node array with
// room for `cap` nodes, per-node costs and subtree counts, object boxes,
// re-split scratch, and the record metadata of the current layout.
struct DynTree {
  int cap = 0;
  int n_objs = 0;
  int next_free = 0;
  bool bounds_valid = false;  // false after a topology-keeping refit
  float* bounds = nullptr;    // 6 per node
  int32_t* child = nullptr;
  int32_t* children = nullptr;
  uint8_t* axis = nullptr;
  uint8_t* lc = nullptr;
  float* costs = nullptr;
  int32_t* n_int = nullptr;  // internal nodes in the subtree
  int32_t* n_obj = nullptr;  // objects in the subtree
  int32_t* parent = nullptr;
  int32_t* arrive = nullptr;
  int32_t* ids = nullptr;
  float* obj_bounds = nullptr;  // 6 per object
  float* obj_cent = nullptr;    // 3 per object
  // re-split scratch: two node slots and one stack entry (3 ints) per object,
  // a leaf using the slots of its own object range
  float* sc_bounds = nullptr;
  int32_t* sc_child = nullptr;
  int32_t* sc_children = nullptr;
  uint8_t* sc_axis = nullptr;
  int32_t* sc_nint = nullptr;
  int32_t* sc_nobj = nullptr;
  int32_t* sc_stack = nullptr;
  // per record child (2 per record, indexed 2 r + side): split size by
  // post-order key, its scanned offset, and the split leaf's own axis/count
  int32_t* slot_count = nullptr;
  int32_t* slot_off = nullptr;
  int32_t* split_axis = nullptr;
  int32_t* split_nint = nullptr;
  // records of the current layout (pre-order), and the level frontiers
  int32_t* rec_node = nullptr;
  int32_t* rec_depth = nullptr;
  int32_t* rec_size = nullptr;
  int32_t* tpos = nullptr;  // the tree's positions before the re-splits
  int32_t* jump[8] = {};     // pointer-jumping buffers (anc, rec, off, dep) x 2
  UpdState* st = nullptr;
  bool layout_host_stale = false;  // host rec_node / level lists behind the device
  void* scan_tmp = nullptr;
  size_t scan_bytes = 0;
  std::vector<void*> allocs;
};

void destroy_dyn_tree(DynTree* d) {
  if (!d) return;
  for (void* p : d->allocs) cudaFree(p);
  delete d;
}

void mark_dyn_bounds_stale(DynTree* d) { d->bounds_valid = false; }

namespace {

constexpr int kBins = 16;

struct DynView {
  float* bounds;
  int32_t* child;
  int32_t* children;
  uint8_t* axis;
  uint8_t* lc;
  float* costs;
  int32_t* n_int;
  int32_t* n_obj;
  int32_t* parent;
  int32_t* arrive;
  int32_t* ids;
  const float* obj_bounds;
  const float* obj_cent;
};

DynView view(const DynTree& d) {
  return DynView{d.bounds, d.child,  d.children, d.axis,   d.lc,         d.costs,   d.n_int,
                 d.n_obj,  d.parent, d.arrive,   d.ids,    d.obj_bounds, d.obj_cent};
}

__device__ __forceinline__ float rmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float rmax(float a, float b) { return a > b ? a : b; }

__device__ __forceinline__ void box_reset(float* b) {
  b[0] = b[1] = b[2] = FLT_MAX;
  b[3] = b[4] = b[5] = -FLT_MAX;
}

__device__ __forceinline__ void box_extend(float* b, const float* o) {
  for (int c = 0; c < 3; ++c) {
    b[c] = rmin(b[c], o[c]);
    b[3 + c] = rmax(b[3 + c], o[3 + c]);
  }
}

// BBox::computeArea: float arithmetic, widened to double
__device__ __forceinline__ double area_d(const float* b) {
  const float dx = __fsub_rn(b[3], b[0]);
  const float dy = __fsub_rn(b[4], b[1]);
  const float dz = __fsub_rn(b[5], b[2]);
  const float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dx, dz));
  return (double)__fmul_rn(2.f, s);
}

__device__ __forceinline__ float area_f(const float* b) { return (float)area_d(b); }

__device__ __forceinline__ int x86_trunc(float x) {
  return (x > -2147483904.f && x < 2147483648.f) ? __float2int_rz(x) : INT_MIN;
}

__device__ __forceinline__ int index_of_max(float a, float b, float c) {
  if (a > b) return a > c ? 0 : 2;
  return b > c ? 1 : 2;
}

// ------------------------------------------------ 1. object boxes -------

__global__ void obj_box_kernel(const float* __restrict__ verts, const uint32_t* __restrict__ idx,
                               int n, float* __restrict__ obj_bounds,
                               float* __restrict__ obj_cent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float tb[6];
  const float* p1 = verts + 3 * (size_t)__ldg(idx + 3 * (size_t)i);
  for (int c = 0; c < 3; ++c) tb[c] = tb[3 + c] = __ldg(p1 + c);
  for (int k = 1; k < 3; ++k) {
    const float* p = verts + 3 * (size_t)__ldg(idx + 3 * (size_t)i + k);
    for (int c = 0; c < 3; ++c) {
      const float x = __ldg(p + c);
      tb[c] = rmin(tb[c], x);
      tb[3 + c] = rmax(tb[3 + c], x);
    }
  }
  float ob[6];
  box_reset(ob);
  box_extend(ob, tb);
  for (int c = 0; c < 6; ++c) obj_bounds[6 * (size_t)i + c] = ob[c];
  for (int c = 0; c < 3; ++c)
    obj_cent[3 * (size_t)i + c] = __fadd_rn(__fmul_rn(ob[3 + c], 0.5f), __fmul_rn(ob[c], 0.5f));
}

// ------------------------------------------------- 2. leaf boxes -------

__device__ void leaf_bounds(DynView V, int c) {
  float b[6];
  box_reset(b);
  const int first = V.child[c], k = V.children[c];
  for (int j = 0; j < k; ++j) box_extend(b, V.obj_bounds + 6 * (size_t)V.ids[first + j]);
  for (int q = 0; q < 6; ++q) V.bounds[6 * (size_t)c + q] = b[q];
  V.axis[c] = 0;
  V.n_int[c] = 0;
  V.n_obj[c] = k;
}

// One thread per (record, side): the child's parent, and its box if a leaf.
__global__ void leaf_pass_kernel(DynView V, const int32_t* __restrict__ rec_node, int n_records,
                                 int32_t* tpos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) tpos[0] = 0;
  if (n_records == 0) {
    if (i == 0) {
      leaf_bounds(V, 0);
      V.parent[0] = -1;
    }
    return;
  }
  if (i >= 2 * n_records) return;
  const int node = rec_node[i >> 1];
  const int c = V.child[node] + (i & 1);
  tpos[i + 1] = c;
  V.parent[c] = node;
  if ((i & 1) == 0) V.arrive[node] = 0;
  if (node == 0 && (i & 1) == 0) V.parent[0] = -1;
  if (V.children[c] != 0) leaf_bounds(V, c);
}

// --------------------------------------------- 3. leaf re-splits -------

struct Part {
  float bl[6], br[6];
  int axis, split;
};

// partition2Objs (DynBVH.cc:2277-2307)
__device__ void partition2(const DynView& V, const float* nb, int b, Part& p) {
  const float node_area = area_f(nb);
  const float left_area = area_f(V.obj_bounds + 6 * (size_t)V.ids[b]);
  const float right_area = area_f(V.obj_bounds + 6 * (size_t)V.ids[b + 1]);
  const float new_cost =
      __fadd_rn(1.f, __fdiv_rn(__fadd_rn(__fmul_rn(left_area, 1.f), __fmul_rn(right_area, 1.f)),
                               node_area));
  if (new_cost < 2.f) {
    p.axis = index_of_max(__fsub_rn(nb[3], nb[0]), __fsub_rn(nb[4], nb[1]),
                          __fsub_rn(nb[5], nb[2]));
    p.split = b + 1;
    if (V.obj_bounds[6 * (size_t)V.ids[b] + p.axis] >
        V.obj_bounds[6 * (size_t)V.ids[b + 1] + p.axis]) {
      const int t = V.ids[b];
      V.ids[b] = V.ids[b + 1];
      V.ids[b + 1] = t;
    }
    for (int q = 0; q < 6; ++q) {
      p.bl[q] = V.obj_bounds[6 * (size_t)V.ids[b] + q];
      p.br[q] = V.obj_bounds[6 * (size_t)V.ids[b + 1] + q];
    }
  } else {
    p.axis = -1;
  }
}

// partitionObjects (DynBVH.cc:1369-1396)
__device__ int partition_objects(const DynView& V, int b, int e, int axis, float pos) {
  int first = b - 1, last = e;
  for (;;) {
    for (++first; first < last; first++)
      if (V.obj_cent[3 * (size_t)V.ids[first] + axis] >= pos) break;
    for (--last; first < last; --last)
      if (V.obj_cent[3 * (size_t)V.ids[last] + axis] < pos) break;
    if (first < last) {
      const int t = V.ids[first];
      V.ids[first] = V.ids[last];
      V.ids[last] = t;
    } else {
      return first;
    }
  }
}

// partitionApproxSAH (DynBVH.cc:2125-2275).  The reference defines
// LONGEST_AXIS (as 0, DynBVH.cc:39), so its #ifdef bins only the centroid
// box's longest axis (BBox::longestAxis, Core/Geometry/BBox.h:123-130).
__device__ void partition_approx(const DynView& V, const float* nb, int b, int e, Part& p) {
  box_reset(p.bl);
  box_reset(p.br);
  const int n = e - b;
  if (n == 1) {
    p.axis = -1;
    p.split = -1;
    return;
  }
  if (n == 2) {
    partition2(V, nb, b, p);
    return;
  }
  float cb[6];
  box_reset(cb);
  for (int i = b; i < e; ++i) {
    const float* c = V.obj_cent + 3 * (size_t)V.ids[i];
    for (int k = 0; k < 3; ++k) {
      cb[k] = rmin(cb[k], c[k]);
      cb[3 + k] = rmax(cb[3 + k], c[k]);
    }
  }
  const float inv_parent_area = __double2float_rn(__ddiv_rn(1.0, area_d(nb)));
  float best_cost = __fmul_rn((float)n, 1.f), best_pos = FLT_MAX;
  int best_axis = -1;
  float width[3], scale[3];
  for (int k = 0; k < 3; ++k) {
    width[k] = __fsub_rn(cb[3 + k], cb[k]);
    scale[k] = __fmul_rn(__fdiv_rn((float)kBins, width[k]), .999f);
  }
  const int a = width[0] > width[1] ? (width[0] > width[2] ? 0 : 2)
                                    : (width[1] > width[2] ? 1 : 2);
  int cnt[kBins];
  float box[kBins][6];
  for (int i = 0; i < kBins; ++i) {
    cnt[i] = 0;
    box_reset(box[i]);
  }
  for (int i = b; i < e; ++i) {
    const int obj = V.ids[i];
    int w = x86_trunc(__fmul_rn(__fsub_rn(V.obj_cent[3 * (size_t)obj + a], cb[a]), scale[a]));
    w = w < 0 ? 0 : w > kBins - 1 ? kBins - 1 : w;
    cnt[w]++;
    box_extend(box[w], V.obj_bounds + 6 * (size_t)obj);
  }
  float la[kBins], ra[kBins];
  int lc[kBins], rc[kBins];
  float lbox[6], rbox[6];
  box_reset(lbox);
  box_reset(rbox);
  int nl = 0, nr = n;
  for (int i = 0; i < kBins; ++i) {
    nl += cnt[i];
    nr -= cnt[i];
    box_extend(lbox, box[i]);
    lc[i] = nl;
    rc[i] = nr;
    la[i] = area_f(lbox);
  }
  for (int i = kBins - 1; i >= 0; --i) {
    ra[i] = (i == kBins - 1) ? FLT_MAX : area_f(rbox);
    box_extend(rbox, box[i]);
  }
  for (int i = 0; i < kBins - 1; ++i) {
    const float cost = __fadd_rn(
        __fmul_rn(__fmul_rn(__fadd_rn(__fmul_rn(la[i], (float)lc[i]), __fmul_rn(ra[i], (float)rc[i])),
                            inv_parent_area),
                  1.f),
        1.f);
    if (cost < best_cost) {
      best_cost = cost;
      best_axis = a;
      best_pos = __fadd_rn(cb[a], __fmul_rn(width[a], __fdiv_rn((float)(i + 1), (float)kBins)));
    }
  }
  p.axis = best_axis;
  if (p.axis == -1) {
    p.split = 0;
    return;
  }
  int middle = partition_objects(V, b, e, p.axis, best_pos);
  if (middle == b || middle == e) middle = b + n / 2;  // n >= 3 here
  for (int i = b; i < middle; ++i) box_extend(p.bl, V.obj_bounds + 6 * (size_t)V.ids[i]);
  for (int i = middle; i < e; ++i) box_extend(p.br, V.obj_bounds + 6 * (size_t)V.ids[i]);
  p.split = middle;
}

struct Scratch {
  float* bounds;
  int32_t* child;
  int32_t* children;
  uint8_t* axis;
  int32_t* nint;
  int32_t* nobj;
  int32_t* stack;
};

// build(leaf, begin, end, useApproximateBuild = true, nodeAlreadyExists =
// true) (DynBVH.cc:1807-1857) into scratch slots 2*begin onward, node
// numbers relative to the first new pair.  Depth-first with an explicit
// stack: the left subtree is finished before the right one starts, so pairs
// are numbered in the reference's allocation order.  Returns the number of
// new nodes; *axis / *nint describe the leaf as an internal node.
__device__ int split_leaf(const DynView& V, int leaf, int b, int e, const Scratch& S, int* axis,
                          int* nint) {
  float* sb = S.bounds + 12 * (size_t)b;
  int32_t* sch = S.child + 2 * (size_t)b;
  int32_t* scn = S.children + 2 * (size_t)b;
  uint8_t* sax = S.axis + 2 * (size_t)b;
  int32_t* sni = S.nint + 2 * (size_t)b;
  int32_t* sno = S.nobj + 2 * (size_t)b;
  int32_t* st = S.stack + 3 * (size_t)b;
  int sp = 0, count = 0;
  st[0] = -1;  // the leaf itself
  st[1] = b;
  st[2] = e;
  sp = 1;
  while (sp > 0) {
    --sp;
    const int node = st[3 * sp], nb = st[3 * sp + 1], ne = st[3 * sp + 2];
    float box[6];
    const float* src = node < 0 ? V.bounds + 6 * (size_t)leaf : sb + 6 * (size_t)node;
    for (int q = 0; q < 6; ++q) box[q] = src[q];
    Part p;
    partition_approx(V, box, nb, ne, p);
    if (p.axis == -1) {
      if (node < 0) return 0;  // the leaf stays a leaf
      sch[node] = nb;
      scn[node] = ne - nb;
      sax[node] = 0;
      // std::sort of the new leaf's object ids (insertion sort: leaves are small)
      for (int i = nb + 1; i < ne; ++i) {
        const int x = V.ids[i];
        int j = i - 1;
        while (j >= nb && V.ids[j] > x) {
          V.ids[j + 1] = V.ids[j];
          --j;
        }
        V.ids[j + 1] = x;
      }
      continue;
    }
    const int spot = count;
    count += 2;
    if (node < 0) {
      *axis = p.axis;
    } else {
      sch[node] = spot;
      scn[node] = 0;
      sax[node] = (uint8_t)p.axis;
    }
    for (int q = 0; q < 6; ++q) {
      sb[6 * (size_t)spot + q] = p.bl[q];
      sb[6 * (size_t)(spot + 1) + q] = p.br[q];
    }
    st[3 * sp] = spot + 1;
    st[3 * sp + 1] = p.split;
    st[3 * sp + 2] = ne;
    st[3 * sp + 3] = spot;
    st[3 * sp + 4] = nb;
    st[3 * sp + 5] = p.split;
    sp += 2;
  }
  // subtree counts, children after parents
  for (int k = count - 1; k >= 0; --k) {
    if (scn[k] != 0) {
      sni[k] = 0;
      sno[k] = scn[k];
    } else {
      const int l = sch[k];
      sni[k] = 1 + sni[l] + sni[l + 1];
      sno[k] = sno[l] + sno[l + 1];
    }
  }
  *nint = 1 + sni[0] + sni[1];
  return count;
}

__device__ __forceinline__ int post_key(const int32_t* rec_depth, const int32_t* rec_size, int r) {
  return r - rec_depth[r] + rec_size[r] - 1;
}

// One thread per (record, side) whose child is a leaf of more than one object.
__global__ void split_kernel(DynView V, Scratch S, const int32_t* __restrict__ rec_node,
                             const int32_t* __restrict__ rec_depth,
                             const int32_t* __restrict__ rec_size, int n_records,
                             int32_t* slot_count, int32_t* split_axis, int32_t* split_nint) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * n_records) return;
  const int r = i >> 1, side = i & 1;
  const int node = rec_node[r];
  const int c = V.child[node] + side;
  const int k = V.children[c];
  int count = 0;
  if (k > 1) {
    int axis = 0, nint = 0;
    const int b = V.child[c];
    count = split_leaf(V, c, b, b + k, S, &axis, &nint);
    split_axis[i] = axis;
    split_nint[i] = nint;
  }
  slot_count[2 * post_key(rec_depth, rec_size, r) + side] = count;
}

// The splits' nodes to their scanned offsets after next_free.
__global__ void relocate_kernel(DynView V, Scratch S, const int32_t* __restrict__ rec_node,
                                const int32_t* __restrict__ rec_depth,
                                const int32_t* __restrict__ rec_size, int n_records,
                                const int32_t* __restrict__ slot_count,
                                const int32_t* __restrict__ slot_off,
                                const int32_t* __restrict__ split_axis,
                                const int32_t* __restrict__ split_nint, int next_free,
                                int cap, UpdState* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * n_records) return;
  const int r = i >> 1, side = i & 1;
  const int key = 2 * post_key(rec_depth, rec_size, r) + side;
  const int count = slot_count[key];
  if (count == 0) return;
  const int base = next_free + slot_off[key];
  if ((long long)base + count > cap) {
    st->error = 1;
    return;
  }
  const int node = rec_node[r];
  const int c = V.child[node] + side;
  const int b = V.child[c];
  const float* sb = S.bounds + 12 * (size_t)b;
  for (int k = 0; k < count; ++k) {
    const int pos = base + k;
    const int j = 2 * b + k;
    for (int q = 0; q < 6; ++q) V.bounds[6 * (size_t)pos + q] = sb[6 * (size_t)k + q];
    const int ch = S.children[j];
    V.children[pos] = ch;
    V.child[pos] = ch != 0 ? S.child[j] : base + S.child[j];
    V.axis[pos] = S.axis[j];
    V.n_int[pos] = S.nint[j];
    V.n_obj[pos] = S.nobj[j];
    // a new leaf's cost; a new internal node keeps whatever the reference's
    // cost array held at that position
    if (ch != 0) V.costs[pos] = __fmul_rn((float)ch, 1.f);
  }
  V.child[c] = base;
  V.children[c] = 0;
  V.axis[c] = (uint8_t)split_axis[i];
  V.n_int[c] = split_nint[i];
}

// ------------------------------------------------- 4. rotations --------
//
// Nodes are handed between threads on different SMs, so every node field is
// read through volatile pointers (L2, never a stale L1 line) and each hand-
// over is one acquire-release atomic on the node's arrival counter: the
// first arrival's writes below the node are released by its increment and
// acquired by the second arrival's, which then reads them.

struct VNodes {
  volatile float* bounds;
  volatile int32_t* child;
  volatile int32_t* children;
  volatile uint8_t* axis;
  volatile uint8_t* lc;
  volatile float* costs;
  volatile int32_t* n_int;
  volatile int32_t* n_obj;

  __device__ void box(int i, float* o) const {
    for (int q = 0; q < 6; ++q) o[q] = bounds[6 * (size_t)i + q];
  }
  __device__ void set_box(int i, const float* b) const {
    for (int q = 0; q < 6; ++q) bounds[6 * (size_t)i + q] = b[q];
  }
  __device__ float area(int i) const {
    float b[6];
    box(i, b);
    return area_f(b);
  }
  __device__ void swap(int a, int b) const {
    for (int q = 0; q < 6; ++q) {
      const float t = bounds[6 * (size_t)a + q];
      bounds[6 * (size_t)a + q] = bounds[6 * (size_t)b + q];
      bounds[6 * (size_t)b + q] = t;
    }
    int t = child[a]; child[a] = child[b]; child[b] = t;
    t = children[a]; children[a] = children[b]; children[b] = t;
    uint8_t u = axis[a]; axis[a] = axis[b]; axis[b] = u;
    u = lc[a]; lc[a] = lc[b]; lc[b] = u;
    const float c = costs[a]; costs[a] = costs[b]; costs[b] = c;
    t = n_int[a]; n_int[a] = n_int[b]; n_int[b] = t;
    t = n_obj[a]; n_obj[a] = n_obj[b]; n_obj[b] = t;
  }
  // Step 3 of rotateNode: the split axis of `parent` guessed from the
  // overlap of children a, b, which are put in order along it
  __device__ void guess_axis(int parent, int a, int b) const {
    float ba[6], bb[6];
    box(a, ba);
    box(b, bb);
    float ov[3];
    for (int k = 0; k < 3; ++k) ov[k] = __fsub_rn(rmax(ba[k], bb[k]), rmin(ba[3 + k], bb[3 + k]));
    const int ax = index_of_max(ov[0], ov[1], ov[2]);
    axis[parent] = (uint8_t)ax;
    if (ba[3 + ax] > bb[3 + ax]) swap(a, b);
  }
  __device__ void counts(int i) const {
    if (children[i] != 0) return;
    const int l = child[i];
    n_int[i] = 1 + n_int[l] + n_int[l + 1];
    n_obj[i] = n_obj[l] + n_obj[l + 1];
  }
};

__device__ __forceinline__ void union_box(const float* a, const float* b, float* o) {
  box_reset(o);
  box_extend(o, a);
  box_extend(o, b);
}

// updateBounds for an internal node (its children done) and rotateNode
// steps 1-3 (the leaf re-splits already applied).
__device__ void rotate_node(const VNodes& V, int id) {
  const int L = V.child[id], R = L + 1;
  float bl[6], br[6], bn[6];
  V.box(L, bl);
  V.box(R, br);
  union_box(bl, br, bn);
  V.set_box(id, bn);
  const int LL = V.child[L], LR = LL + 1, RL = V.child[R], RR = RL + 1;
  const bool l_leaf = V.children[L] != 0, r_leaf = V.children[R] != 0;
  const float node_area = area_f(bn);
  const float left_area = area_f(bl);
  const float right_area = area_f(br);
  const float cL = V.costs[L], cR = V.costs[R];
  float ll_area = 0.f, lr_area = 0.f, rl_area = 0.f, rr_area = 0.f;
  float cLL = 0.f, cLR = 0.f, cRL = 0.f, cRR = 0.f;
  float box_a[6], box_b[6];
  float area_a = 0.f, area_b = 0.f;
  int best = 0;
  float best_cost = __fadd_rn(__fadd_rn(__fmul_rn(node_area, 1.f), __fmul_rn(left_area, cL)),
                              __fmul_rn(right_area, cR));
  float bll[6], blr[6], brl[6], brr[6];
  if (!l_leaf) {
    V.box(LL, bll);
    V.box(LR, blr);
    cLL = V.costs[LL];
    cLR = V.costs[LR];
    ll_area = area_f(bll);
    lr_area = area_f(blr);
    const float partial = __fadd_rn(
        __fadd_rn(__fadd_rn(__fmul_rn(node_area, 1.f), __fmul_rn(right_area, cR)),
                  __fmul_rn(lr_area, cLR)),
        __fmul_rn(ll_area, cLL));
    float b1[6], b2[6];
    for (int q = 0; q < 6; ++q) b1[q] = b2[q] = br[q];
    box_extend(b1, blr);  // (1) R <-> LL
    const float a1 = area_f(b1);
    const float u1 = __fadd_rn(__fmul_rn(a1, 1.f), partial);
    if (u1 < best_cost) {
      best = 1; best_cost = u1; area_a = a1;
      for (int q = 0; q < 6; ++q) box_a[q] = b1[q];
    }
    box_extend(b2, bll);  // (2) R <-> LR
    const float a2 = area_f(b2);
    const float u2 = __fadd_rn(__fmul_rn(a2, 1.f), partial);
    if (u2 < best_cost) {
      best = 2; best_cost = u2; area_a = a2;
      for (int q = 0; q < 6; ++q) box_a[q] = b2[q];
    }
  }
  if (!r_leaf) {
    V.box(RL, brl);
    V.box(RR, brr);
    cRL = V.costs[RL];
    cRR = V.costs[RR];
    rl_area = area_f(brl);
    rr_area = area_f(brr);
    const float partial = __fadd_rn(
        __fadd_rn(__fadd_rn(__fmul_rn(node_area, 1.f), __fmul_rn(left_area, cL)),
                  __fmul_rn(rr_area, cRR)),
        __fmul_rn(rl_area, cRL));
    float b3[6], b4[6];
    for (int q = 0; q < 6; ++q) b3[q] = b4[q] = bl[q];
    box_extend(b3, brr);  // (3) L <-> RL
    const float a3 = area_f(b3);
    const float u3 = __fadd_rn(__fmul_rn(a3, 1.f), partial);
    if (u3 < best_cost) {
      best = 3; best_cost = u3; area_a = a3;
      for (int q = 0; q < 6; ++q) box_a[q] = b3[q];
    }
    box_extend(b4, brl);  // (4) L <-> RR
    const float a4 = area_f(b4);
    const float u4 = __fadd_rn(__fmul_rn(a4, 1.f), partial);
    if (u4 < best_cost) {
      best = 4; best_cost = u4; area_a = a4;
      for (int q = 0; q < 6; ++q) box_a[q] = b4[q];
    }
    if (!l_leaf) {
      const float partial2 = __fadd_rn(
          __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(node_area, 1.f), __fmul_rn(ll_area, cLL)),
                              __fmul_rn(lr_area, cLR)),
                    __fmul_rn(rl_area, cRL)),
          __fmul_rn(rr_area, cRR));
      float b5l[6], b5r[6], b6l[6], b6r[6];
      for (int q = 0; q < 6; ++q) {
        b5l[q] = b6l[q] = bll[q];
        b5r[q] = blr[q];
        b6r[q] = brl[q];
      }
      box_extend(b5l, brl);  // (5) LR <-> RL
      box_extend(b5r, brr);
      const float a5l = area_f(b5l), a5r = area_f(b5r);
      const float u5 = __fadd_rn(__fmul_rn(__fadd_rn(a5l, a5r), 1.f), partial2);
      if (u5 < best_cost) {
        best = 5; best_cost = u5; area_a = a5l; area_b = a5r;
        for (int q = 0; q < 6; ++q) {
          box_a[q] = b5l[q];
          box_b[q] = b5r[q];
        }
      }
      box_extend(b6l, brr);  // (6) LR <-> RR
      box_extend(b6r, blr);
      const float a6l = area_f(b6l), a6r = area_f(b6r);
      const float u6 = __fadd_rn(__fmul_rn(__fadd_rn(a6l, a6r), 1.f), partial2);
      if (u6 < best_cost) {
        best = 6; best_cost = u6; area_a = a6l; area_b = a6r;
        for (int q = 0; q < 6; ++q) {
          box_a[q] = b6l[q];
          box_b[q] = b6r[q];
        }
      }
    }
  }
  V.costs[id] = __fdiv_rn(best_cost, node_area);
  if (best != 0) {
    const float inv_a = __fdiv_rn(1.f, area_a);
    switch (best) {
      case 1:
        V.set_box(L, box_a);
        V.costs[L] = __fadd_rn(1.f, __fmul_rn(__fadd_rn(__fmul_rn(lr_area, cLR),
                                                        __fmul_rn(right_area, cR)), inv_a));
        V.swap(LL, R);
        break;
      case 2:
        V.set_box(L, box_a);
        V.costs[L] = __fadd_rn(1.f, __fmul_rn(__fadd_rn(__fmul_rn(ll_area, cLL),
                                                        __fmul_rn(right_area, cR)), inv_a));
        V.swap(LR, R);
        break;
      case 3:
        V.set_box(R, box_a);
        V.costs[R] = __fadd_rn(1.f, __fmul_rn(__fadd_rn(__fmul_rn(rr_area, cRR),
                                                        __fmul_rn(left_area, cL)), inv_a));
        V.swap(RL, L);
        break;
      case 4:
        V.set_box(R, box_a);
        V.costs[R] = __fadd_rn(1.f, __fmul_rn(__fadd_rn(__fmul_rn(rl_area, cRL),
                                                        __fmul_rn(left_area, cL)), inv_a));
        V.swap(RR, L);
        break;
      case 5:
        V.set_box(L, box_a);
        V.set_box(R, box_b);
        V.costs[L] = __fadd_rn(1.f, __fmul_rn(__fadd_rn(__fmul_rn(ll_area, cLL),
                                                        __fmul_rn(rl_area, cRL)), inv_a));
        V.costs[R] = __fadd_rn(1.f, __fdiv_rn(__fadd_rn(__fmul_rn(lr_area, cLR),
                                                        __fmul_rn(rr_area, cRR)), area_b));
        V.swap(LR, RL);
        break;
      default:
        V.set_box(L, box_a);
        V.set_box(R, box_b);
        V.costs[L] = __fadd_rn(1.f, __fmul_rn(__fadd_rn(__fmul_rn(ll_area, cLL),
                                                        __fmul_rn(rr_area, cRR)), inv_a));
        V.costs[R] = __fadd_rn(1.f, __fdiv_rn(__fadd_rn(__fmul_rn(lr_area, cLR),
                                                        __fmul_rn(rl_area, cRL)), area_b));
        V.swap(LR, RR);
        break;
    }
    if (best <= 2 || best >= 5) V.guess_axis(L, LL, LR);
    if (best >= 3) V.guess_axis(R, RL, RR);
    V.guess_axis(id, L, R);
  }
  V.counts(L);
  V.counts(R);
  V.counts(id);
}

// One thread per original leaf climbs to the root; the second arrival at a
// node rotates it and climbs on.
__global__ void rotate_kernel(DynView D, const float4* __restrict__ recs,
                              const int32_t* __restrict__ rec_node, int n_records) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * n_records) return;
  const int4 q3 = reinterpret_cast<const int4*>(recs)[4 * (size_t)(i >> 1) + 3];
  const int ref = (i & 1) ? q3.y : q3.x;
  if (ref >= 0) return;  // an internal child climbs from its own leaves
  const VNodes V{D.bounds, D.child, D.children, D.axis, D.lc, D.costs, D.n_int, D.n_obj};
  volatile int32_t* parent = D.parent;
  int node = rec_node[i >> 1];
  while (node >= 0) {
    // one acquire-release arrival: releases this thread's writes below
    // `node` and, for the second arrival, acquires the sibling's
    int first;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                 : "=r"(first)
                 : "l"(D.arrive + node)
                 : "memory");
    if (first == 0) return;
    rotate_node(V, node);
    node = parent[node];
  }
}

// ------------------------------------------------- 5. relayout ---------
//
// The records are numbered in pre-order of the internal nodes and the
// leaves' objects placed in pre-order, both known from the subtree counts:
// a node's record number is the sum over the edges from the root of
// 1 (+ the internal nodes of the left sibling for a right child), its first
// object the sum of the left siblings' object counts.  Those sums along the
// path to the root are formed by pointer jumping (each round adds the
// ancestor's partial sum and jumps to the ancestor's ancestor), so the whole
// layout takes a fixed number of launches and no host round trip.
// The tree's positions: 0, the children of the records before the update,
// and the pairs the re-splits added (next_free before .. after).

struct Jump {
  int32_t* anc;
  int32_t* rec;
  int32_t* off;
  int32_t* dep;
};

__device__ __forceinline__ int tree_position(int i, const int32_t* __restrict__ tpos, int m_old,
                                             int nf_old, const UpdState* st) {
  if (i < m_old) return tpos[i];
  const int p = nf_old + (i - m_old);
  return p < st->next_free ? p : -1;
}

__global__ void init_state_kernel(UpdState* st, int next_free) {
  st->next_free = next_free;
  st->error = 0;
  st->n_records = 0;
  st->depth = 0;
}

// The re-splits' pairs land after next_free; advance it (one thread).
__global__ void advance_kernel(const int32_t* __restrict__ slot_count,
                               const int32_t* __restrict__ slot_off, int n_slots, int cap,
                               UpdState* st) {
  const long long total =
      n_slots > 0 ? (long long)slot_off[n_slots - 1] + slot_count[n_slots - 1] : 0;
  if (st->next_free + total > cap) {
    st->error = 1;
    return;
  }
  st->next_free += (int)total;
}

__global__ void parent_pass_kernel(DynView V, const int32_t* __restrict__ tpos, int m_old,
                                   int nf_old, const UpdState* st, int m_max) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m_max) return;
  const int p = tree_position(i, tpos, m_old, nf_old, st);
  if (p < 0) return;
  if (p == 0) V.parent[0] = -1;
  if (V.children[p] == 0) {
    const int c = V.child[p];
    V.parent[c] = p;
    V.parent[c + 1] = p;
  }
}

__global__ void jump_init_kernel(DynView V, const int32_t* __restrict__ tpos, int m_old,
                                 int nf_old, const UpdState* st, int m_max, Jump J) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m_max) return;
  const int p = tree_position(i, tpos, m_old, nf_old, st);
  if (p < 0) return;
  if (p == 0) {
    J.anc[0] = -1;
    J.rec[0] = J.off[0] = J.dep[0] = 0;
    return;
  }
  const int y = V.parent[p];
  const int left = V.child[y];
  const bool right = p == left + 1;
  J.anc[p] = y;
  J.rec[p] = 1 + (right ? V.n_int[left] : 0);
  J.off[p] = right ? V.n_obj[left] : 0;
  J.dep[p] = 1;
}

__global__ void jump_kernel(const int32_t* __restrict__ tpos, int m_old, int nf_old,
                            const UpdState* st, int m_max, Jump S, Jump D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m_max) return;
  const int p = tree_position(i, tpos, m_old, nf_old, st);
  if (p < 0) return;
  const int a = S.anc[p];
  if (a < 0) {
    D.anc[p] = -1;
    D.rec[p] = S.rec[p];
    D.off[p] = S.off[p];
    D.dep[p] = S.dep[p];
  } else {
    D.anc[p] = S.anc[a];
    D.rec[p] = S.rec[p] + S.rec[a];
    D.off[p] = S.off[p] + S.off[a];
    D.dep[p] = S.dep[p] + S.dep[a];
  }
}

// Records, leaf object order, depth and root box from the summed paths.
__global__ void emit_kernel(DynView V, const int32_t* __restrict__ tpos, int m_old, int nf_old,
                            UpdState* st, int m_max, Jump J, float4* recs, int rec_cap,
                            int32_t* perm, int n_objs, int32_t* rec_node, int32_t* rec_depth,
                            int32_t* rec_size) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m_max) return;
  const int p = tree_position(i, tpos, m_old, nf_old, st);
  if (p < 0) return;
  if (J.anc[p] >= 0) {  // deeper than the rounds reach
    st->error = 2;
    return;
  }
  const int rec = J.rec[p], off = J.off[p], dep = J.dep[p];
  if (p == 0) {
    st->n_records = V.children[0] == 0 ? V.n_int[0] : 0;
    for (int q = 0; q < 6; ++q) st->root[q] = V.bounds[q];
  }
  const int k = V.children[p];
  if (k != 0) {
    atomicMax(&st->depth, dep);
    const int first = V.child[p];
    for (int j = 0; j < k; ++j) {
      if (off + j >= n_objs) {
        st->error = 3;
        break;
      }
      const int obj = V.ids[first + j];
      perm[off + j] = j == k - 1 ? (int32_t)(obj | 0x80000000u) : obj;
    }
    return;
  }
  if (rec >= rec_cap) {
    st->error = 3;
    return;
  }
  const int L = V.child[p], R = L + 1;
  const int ref_l = V.children[L] != 0 ? ~off : rec + 1;
  const int ref_r = V.children[R] != 0 ? ~(off + V.n_obj[L]) : rec + 1 + V.n_int[L];
  const float* bl = V.bounds + 6 * (size_t)L;
  const float* br = V.bounds + 6 * (size_t)R;
  float4* q = recs + 4 * (size_t)rec;
  q[0] = make_float4(bl[0], bl[1], bl[2], bl[3]);
  q[1] = make_float4(bl[4], bl[5], br[0], br[1]);
  q[2] = make_float4(br[2], br[3], br[4], br[5]);
  const int meta = (V.axis[p] & 3) | ((V.lc[p] & 1) << 2);
  reinterpret_cast<int4*>(q)[3] = make_int4(ref_l, ref_r, meta, 0);
  rec_node[rec] = p;
  rec_depth[rec] = dep;
  rec_size[rec] = V.n_int[p];
}

inline int blocks(long long n, int t) { return (int)std::max<long long>(1, (n + t - 1) / t); }

}  // namespace

// ------------------------------------------------------------ host -----

namespace {

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string("rotating update: ") + what + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? RQ_ERR_OOM : RQ_ERR_CUDA;
}

template <typename T>
cudaError_t dalloc(DynTree* d, T** p, size_t count) {
  void* q = nullptr;
  const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e == cudaSuccess) {
    d->allocs.push_back(q);
    *p = static_cast<T*>(q);
  }
  return e;
}

#define DY_CUDA(call, what)                    \
  do {                                         \
    const cudaError_t e_ = (call);             \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

// Grows the record buffers to hold any tree over the scene's objects.
int ensure_record_capacity(Scene* s) {
  const int need = std::max(s->n_tris - 1, 1);
  if (s->rec_capacity >= need) return RQ_OK;
  float4* nodes = nullptr;
  int32_t* levels = nullptr;
  DY_CUDA(cudaMalloc(&nodes, (size_t)need * 4 * sizeof(float4)), "record buffer");
  cudaError_t e = cudaMalloc(&levels, (size_t)need * sizeof(int32_t));
  if (e == cudaSuccess && s->n_records > 0)
    e = cudaMemcpy(nodes, s->d_nodes, (size_t)s->n_records * 4 * sizeof(float4),
                   cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess && s->n_records > 0)
    e = cudaMemcpy(levels, s->d_level_recs, (size_t)s->n_records * sizeof(int32_t),
                   cudaMemcpyDeviceToDevice);
  if (e != cudaSuccess) {
    cudaFree(nodes);
    cudaFree(levels);
    return cuda_fail(e, "record buffer");
  }
  cudaFree(s->d_nodes);
  cudaFree(s->d_level_recs);
  s->d_nodes = nodes;
  s->d_level_recs = levels;
  s->rec_capacity = need;
  return RQ_OK;
}

// Device node arrays from the host tree (first rotating update), or only
// their boxes (after a topology-keeping refit).
int dyn_sync(Scene* s) {
  DynTree* d = s->dyn;
  if (d && d->bounds_valid) return RQ_OK;
  int rc = s->refresh_tree();
  if (rc != RQ_OK) return rc;
  const HostTree& t = s->tree;
  const int nn = (int)t.children.size();
  if (d) {
    DY_CUDA(cudaMemcpy(d->bounds, t.bounds.data(), (size_t)nn * 6 * sizeof(float),
                       cudaMemcpyHostToDevice), "boxes");
    d->bounds_valid = true;
    return RQ_OK;
  }
  rc = ensure_record_capacity(s);
  if (rc != RQ_OK) return rc;
  d = new DynTree();
  const int N = s->n_tris;
  const int I = s->n_records;
  d->n_objs = N;
  d->next_free = s->tree_next_free;
  d->cap = std::max({2 * N, d->next_free + 2 * std::max(N - 1 - I, 0), nn});
  const size_t cap = d->cap, n = std::max(N, 1), nr = std::max(N - 1, 1);
  cudaError_t e = cudaSuccess;
  auto A = [&](auto** p, size_t count) {
    if (e == cudaSuccess) e = dalloc(d, p, count);
  };
  A(&d->bounds, 6 * cap);
  A(&d->child, cap);
  A(&d->children, cap);
  A(&d->axis, cap);
  A(&d->lc, cap);
  A(&d->costs, cap);
  A(&d->n_int, cap);
  A(&d->n_obj, cap);
  A(&d->parent, cap);
  A(&d->arrive, cap);
  A(&d->ids, n);
  A(&d->obj_bounds, 6 * n);
  A(&d->obj_cent, 3 * n);
  A(&d->sc_bounds, 12 * n);
  A(&d->sc_child, 2 * n);
  A(&d->sc_children, 2 * n);
  A(&d->sc_axis, 2 * n);
  A(&d->sc_nint, 2 * n);
  A(&d->sc_nobj, 2 * n);
  A(&d->sc_stack, 3 * n);
  A(&d->slot_count, 2 * nr);
  A(&d->slot_off, 2 * nr);
  A(&d->split_axis, 2 * nr);
  A(&d->split_nint, 2 * nr);
  A(&d->rec_node, nr);
  A(&d->rec_depth, nr);
  A(&d->rec_size, nr);
  A(&d->tpos, 2 * n);
  for (int k = 0; k < 8; ++k) A(&d->jump[k], cap);
  A(&d->st, 1);
  if (e == cudaSuccess)
    e = cub::DeviceScan::ExclusiveSum(nullptr, d->scan_bytes, d->slot_count, d->slot_off,
                                      (int)(2 * nr));
  if (e == cudaSuccess) A(reinterpret_cast<uint8_t**>(&d->scan_tmp), d->scan_bytes);
  // contents
  std::vector<float> costs(cap, 0.f);
  std::copy(s->tree_costs.begin(), s->tree_costs.end(), costs.begin());
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (e == cudaSuccess && bytes > 0) e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  };
  if (e == cudaSuccess) e = cudaMemset(d->bounds, 0, 6 * cap * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(d->child, 0, cap * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemset(d->children, 0, cap * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemset(d->axis, 0, cap);
  if (e == cudaSuccess) e = cudaMemset(d->lc, 0, cap);
  up(d->bounds, t.bounds.data(), (size_t)nn * 6 * sizeof(float));
  up(d->child, t.child.data(), (size_t)nn * sizeof(int32_t));
  up(d->children, t.children.data(), (size_t)nn * sizeof(int32_t));
  up(d->axis, t.axis.data(), (size_t)nn);
  up(d->lc, t.left_cheaper.data(), (size_t)nn);
  up(d->costs, costs.data(), cap * sizeof(float));
  up(d->ids, t.ids.data(), (size_t)N * sizeof(int32_t));
  up(d->rec_node, s->rec_node.data(), (size_t)I * sizeof(int32_t));
  up(d->rec_depth, s->rec_depth.data(), (size_t)I * sizeof(int32_t));
  up(d->rec_size, s->rec_size.data(), (size_t)I * sizeof(int32_t));
  if (e != cudaSuccess) {
    destroy_dyn_tree(d);
    return cuda_fail(e, "device tree");
  }
  d->bounds_valid = true;
  s->dyn = d;
  return RQ_OK;
}

}  // namespace

// The rotating update on the scene's device vertices (already uploaded).
int rotate_update(Scene* s) {
  if (s->n_tris < 1) return fail(RQ_ERR_STATE, "scene has no triangles");
  if ((int)s->tree.ids.size() != s->n_tris || s->n_leaf_tris != s->n_tris)
    return fail(RQ_ERR_STATE,
                "the rotating update needs a tree whose leaves hold every triangle once");
  int rc = dyn_sync(s);
  if (rc != RQ_OK) return rc;
  DynTree& d = *s->dyn;
  const DynView V = view(d);
  const int N = s->n_tris;
  const int T = 256;
  const int nrec = s->n_records;
  const int nf_old = d.next_free;
  init_state_kernel<<<1, 1>>>(d.st, nf_old);
  obj_box_kernel<<<blocks(N, T), T>>>(s->d_verts, s->d_idx, N, d.obj_bounds, d.obj_cent);
  leaf_pass_kernel<<<blocks(2LL * nrec, T), T>>>(V, d.rec_node, nrec, d.tpos);
  DY_CUDA(cudaGetLastError(), "leaf boxes");
  if (nrec > 0) {
    const Scratch S{d.sc_bounds, d.sc_child, d.sc_children, d.sc_axis,
                    d.sc_nint,   d.sc_nobj,  d.sc_stack};
    split_kernel<<<blocks(2LL * nrec, 128), 128>>>(V, S, d.rec_node, d.rec_depth, d.rec_size,
                                                   nrec, d.slot_count, d.split_axis,
                                                   d.split_nint);
    DY_CUDA(cudaGetLastError(), "leaf re-splits");
    size_t bytes = d.scan_bytes;
    DY_CUDA(cub::DeviceScan::ExclusiveSum(d.scan_tmp, bytes, d.slot_count, d.slot_off,
                                          2 * nrec),
            "split offsets");
    relocate_kernel<<<blocks(2LL * nrec, T), T>>>(V, S, d.rec_node, d.rec_depth, d.rec_size,
                                                  nrec, d.slot_count, d.slot_off, d.split_axis,
                                                  d.split_nint, nf_old, d.cap, d.st);
    advance_kernel<<<1, 1>>>(d.slot_count, d.slot_off, 2 * nrec, d.cap, d.st);
    rotate_kernel<<<blocks(2LL * nrec, T), T>>>(V, s->d_nodes, d.rec_node, nrec);
    DY_CUDA(cudaGetLastError(), "rotations");
  }
  // layout of the updated tree: the positions before the re-splits and the
  // pairs they added (at most 2 (N - 1 - records) more)
  const int m_old = 2 * nrec + 1;
  const int m_max = m_old + 2 * std::max(N - 1 - nrec, 0);
  parent_pass_kernel<<<blocks(m_max, T), T>>>(V, d.tpos, m_old, nf_old, d.st, m_max);
  Jump J[2] = {{d.jump[0], d.jump[1], d.jump[2], d.jump[3]},
               {d.jump[4], d.jump[5], d.jump[6], d.jump[7]}};
  jump_init_kernel<<<blocks(m_max, T), T>>>(V, d.tpos, m_old, nf_old, d.st, m_max, J[0]);
  int cur = 0;
  for (int round = 0; (1 << round) < kMaxDepth; ++round) {
    jump_kernel<<<blocks(m_max, T), T>>>(d.tpos, m_old, nf_old, d.st, m_max, J[cur],
                                         J[cur ^ 1]);
    cur ^= 1;
  }
  emit_kernel<<<blocks(m_max, T), T>>>(V, d.tpos, m_old, nf_old, d.st, m_max, J[cur],
                                       s->d_nodes, s->rec_capacity, s->d_perm, N, d.rec_node,
                                       d.rec_depth, d.rec_size);
  DY_CUDA(cudaGetLastError(), "relayout");
  DY_CUDA(launch_tri_setup(s->tri_kind, s->d_verts, s->d_idx, s->d_perm, N, s->d_tris, 0),
          "triangle records");
  UpdState out;
  DY_CUDA(cudaMemcpy(&out, d.st, sizeof(out), cudaMemcpyDeviceToHost), "update state");
  if (out.error != 0) {
    // the device tree is no longer consistent: drop it
    s->free_tree();
    return fail(out.error == 2 ? RQ_ERR_CAPACITY : RQ_ERR_STATE,
                out.error == 1   ? "leaf re-splits need more nodes than the tree holds"
                : out.error == 2 ? "updated tree is deeper than the traversal stack limit"
                                 : "updated tree's records exceed the record buffer");
  }
  d.next_free = out.next_free;
  d.layout_host_stale = true;
  s->n_records = out.n_records;
  s->n_leaves = out.n_records + 1;
  s->root_ref = out.n_records > 0 ? 0 : ~0;
  for (int c = 0; c < 3; ++c) {
    s->root_lo[c] = out.root[c];
    s->root_hi[c] = out.root[3 + c];
  }
  s->depth = std::max(out.depth, 1);
  s->tree_stale = true;
  s->tree_from_dyn = true;
  ++s->generation;
  return RQ_OK;
}

// After rotating updates the host's record list and the records grouped by
// level (the topology-keeping refit's bottom-up order) are brought up to
// date only when a refit needs them.
int sync_layout_host(Scene* s) {
  if (!s->dyn || !s->dyn->layout_host_stale) return RQ_OK;
  DynTree& d = *s->dyn;
  const int n = s->n_records;
  std::vector<int32_t> rn((size_t)n), rd((size_t)n);
  if (n > 0) {
    DY_CUDA(cudaMemcpy(rn.data(), d.rec_node, (size_t)n * sizeof(int32_t),
                       cudaMemcpyDeviceToHost),
            "records");
    DY_CUDA(cudaMemcpy(rd.data(), d.rec_depth, (size_t)n * sizeof(int32_t),
                       cudaMemcpyDeviceToHost),
            "records");
  }
  int maxd = 0;
  for (int x : rd) maxd = std::max(maxd, x);
  std::vector<int> count(maxd + 1, 0), start(maxd + 2, 0);
  for (int x : rd) ++count[x];
  for (int x = maxd; x >= 0; --x) start[maxd - x + 1] = start[maxd - x] + count[x];
  std::vector<int> fill(start.begin(), start.end() - 1);
  std::vector<int32_t> by_level((size_t)n);
  for (int r = 0; r < n; ++r) by_level[fill[maxd - rd[r]]++] = r;
  if (n > 0)
    DY_CUDA(cudaMemcpy(s->d_level_recs, by_level.data(), (size_t)n * sizeof(int32_t),
                       cudaMemcpyHostToDevice),
            "levels");
  s->level_offsets.assign(start.begin(), start.end());
  if (n == 0) s->level_offsets.assign(1, 0);
  s->rec_node.swap(rn);
  d.layout_host_stale = false;
  return RQ_OK;
}

// The host tree from the device arrays (export, SAH cost).
int refresh_tree_from_dyn(const Scene* s) {
  const DynTree& d = *s->dyn;
  HostTree& t = s->tree;
  const size_t n = d.next_free;
  t.bounds.resize(6 * n);
  t.child.resize(n);
  t.children.resize(n);
  t.axis.resize(n);
  t.left_cheaper.resize(n);
  t.ids.resize(d.n_objs);
  cudaError_t e = cudaMemcpy(t.bounds.data(), d.bounds, 6 * n * sizeof(float),
                             cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(t.child.data(), d.child, n * sizeof(int32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(t.children.data(), d.children, n * sizeof(int32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(t.axis.data(), d.axis, n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(t.left_cheaper.data(), d.lc, n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(t.ids.data(), d.ids, (size_t)d.n_objs * sizeof(int32_t),
                   cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "reading the tree");
  return RQ_OK;
}

// The per-node costs and next free node the next rotating update starts
// from (count = next free node), for checks against the reference.
int dyn_state(const Scene* s, float* costs, int cap, int* next_free) {
  if (!s->dyn) return fail(RQ_ERR_STATE, "no rotating update has run on this scene");
  const DynTree& d = *s->dyn;
  *next_free = d.next_free;
  if (!costs) return RQ_OK;
  if (cap < d.next_free) return fail(RQ_ERR_CAPACITY, "cost array too small");
  DY_CUDA(cudaMemcpy(costs, d.costs, (size_t)d.next_free * sizeof(float),
                     cudaMemcpyDeviceToHost),
          "costs");
  return RQ_OK;
}

}  // namespace rq

extern "C" int rq_scene_update_state(const rq_scene* scene, float* costs, int capacity,
                                     int* next_free) {
  using namespace rq;
  if (!scene || !next_free) {
    set_error("NULL argument");
    return RQ_ERR_ARG;
  }
  if (cudaSetDevice(scene->device) != cudaSuccess) {
    set_error("cudaSetDevice");
    return RQ_ERR_CUDA;
  }
  return dyn_state(scene, costs, capacity, next_free);
}
