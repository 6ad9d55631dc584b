/*
 * Test infrastructure, not product code: the CPU restatement of the
 * reference's DynBVH::update for an animated mesh, used only by tests/ to
 * check rq_scene_update_vertices_ex(..., RQ_UPDATE_ROTATE).
 *
 * Restated, single-threaded (DynBVH::update(0, 1)), in the reference's
 * float operation order (compile with -ffp-contract=off):
 *
 *   object boxes      parallelUpdateBounds (Model/Groups/DynBVH.cc:2012-2031):
 *                     obj_bounds = reset + MeshTriangle::computeBounds
 *                     (Mesh::getBBox, Model/Groups/Mesh.cc:228-237),
 *                     obj_centroids = BBox::center (Core/Geometry/BBox.h:66-68,
 *                     Interpolate with a float weight, Core/Math/MiscMath.h:135-139)
 *   bounds            updateBounds (DynBVH.cc:2068-2123): post-order; a
 *                     leaf's box is the union of its objects' boxes (axis
 *                     reset to 0), an internal node's the union of its
 *                     children's, then rotateNode
 *   rotations         rotateNode (DynBVH.cc:3051-3348), Kopta et al. 2012:
 *                     leaf children with more than one object are re-split
 *                     by the approximate build, then the best of six
 *                     rotations by SAH cost is applied, costs updated and
 *                     the split axes guessed again
 *   leaf re-split     build (DynBVH.cc:1807-1857) with partitionApproxSAH
 *                     (2125-2275, 16 bins on the centroid box's longest
 *                     axis), partition2Objs
 *                     (2277-2307) and partitionObjects (1369-1396)
 *   costs             computeCost<true> (DynBVH.cc:3389-3416), the state a
 *                     rebuild leaves for the first update
 *
 * Min/Max are the reference's ternaries (Core/Math/MinMax.h:83-91), boxes
 * start from [FLT_MAX, -FLT_MAX] (BBox::reset), BBox::computeArea is
 * evaluated in float and widened to double, so 1.0f / area is a double
 * division rounded to float where the reference writes it that way.
 * The reference's int(float) conversion is x86's cvttss2si: NaN and
 * out-of-range values give INT_MIN.
 *
 * Tree: the reference's node array field by field (bounds[6*i] = min xyz,
 * max xyz; child; children, leaf iff != 0; axis; isLeftCheaper), the per-node
 * costs, object_ids and the next free node (DynBVH::nextFree).  isLargeSubtree
 * and subtree_size only steer the reference's multi-threaded update and are
 * not kept.
 */
#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  float* bounds;
  int* child;
  int* children;
  unsigned char* axis;
  unsigned char* left_cheaper;
  float* costs;
  int* ids;
  int cap;
  int next_free;
  float* obj_bounds; /* 6 per object */
  float* obj_cent;   /* 3 per object */
  int overflow;
} UTree;

typedef struct {
  float bl[6], br[6];
  int axis, split;
} Part;

static float ref_min(float a, float b) { return a < b ? a : b; }
static float ref_max(float a, float b) { return a > b ? a : b; }

static void box_reset(float* b) {
  b[0] = b[1] = b[2] = FLT_MAX;
  b[3] = b[4] = b[5] = -FLT_MAX;
}

static void box_extend(float* b, const float* o) {
  for (int c = 0; c < 3; ++c) {
    b[c] = ref_min(b[c], o[c]);
    b[3 + c] = ref_max(b[3 + c], o[3 + c]);
  }
}

static void box_copy(float* d, const float* s) { memcpy(d, s, 6 * sizeof(float)); }

/* BBox::computeArea: float arithmetic, returned as double */
static double box_area_d(const float* b) {
  float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
  float s = dx * dy + dy * dz + dx * dz;
  return (double)(2 * s);
}

static float area_f(const float* b) { return (float)box_area_d(b); }

static int x86_trunc(float x) {
  if (!(x > -2147483904.f && x < 2147483648.f)) return INT32_MIN;
  return (int)x;
}

/* Vector::indexOfMaxComponent (Core/Geometry/Vector.h:382-394): a tie goes
   to the later component */
static int index_of_max(const float* v) {
  if (v[0] > v[1]) return v[0] > v[2] ? 0 : 2;
  return v[1] > v[2] ? 1 : 2;
}

static void node_swap(UTree* T, int a, int b) {
  float tb[6];
  box_copy(tb, T->bounds + 6 * (size_t)a);
  box_copy(T->bounds + 6 * (size_t)a, T->bounds + 6 * (size_t)b);
  box_copy(T->bounds + 6 * (size_t)b, tb);
  int ti = T->child[a]; T->child[a] = T->child[b]; T->child[b] = ti;
  ti = T->children[a]; T->children[a] = T->children[b]; T->children[b] = ti;
  unsigned char tc = T->axis[a]; T->axis[a] = T->axis[b]; T->axis[b] = tc;
  tc = T->left_cheaper[a]; T->left_cheaper[a] = T->left_cheaper[b]; T->left_cheaper[b] = tc;
  float tf = T->costs[a]; T->costs[a] = T->costs[b]; T->costs[b] = tf;
}

/* --------------------------------------------------------- partitions --- */

static Part partition2(UTree* T, int node, int b) {
  Part p;
  box_reset(p.bl);
  box_reset(p.br);
  const float* nb = T->bounds + 6 * (size_t)node;
  const float node_area = area_f(nb);
  const float left_area = area_f(T->obj_bounds + 6 * (size_t)T->ids[b]);
  const float right_area = area_f(T->obj_bounds + 6 * (size_t)T->ids[b + 1]);
  const float leaf_cost = 1.f * 2;
  const float new_cost = 1.f + (left_area * 1.f + right_area * 1.f) / node_area;
  if (new_cost < leaf_cost) {
    float diag[3] = {nb[3] - nb[0], nb[4] - nb[1], nb[5] - nb[2]};
    p.axis = index_of_max(diag);
    p.split = b + 1;
    if (T->obj_bounds[6 * (size_t)T->ids[b] + p.axis] >
        T->obj_bounds[6 * (size_t)T->ids[b + 1] + p.axis]) {
      int t = T->ids[b];
      T->ids[b] = T->ids[b + 1];
      T->ids[b + 1] = t;
    }
    box_copy(p.bl, T->obj_bounds + 6 * (size_t)T->ids[b]);
    box_copy(p.br, T->obj_bounds + 6 * (size_t)T->ids[b + 1]);
  } else {
    p.axis = -1;
  }
  return p;
}

static int partition_objects(UTree* T, int b, int e, int axis, float position) {
  int first = b - 1, last = e;
  for (;;) {
    for (++first; first < last; first++)
      if (T->obj_cent[3 * (size_t)T->ids[first] + axis] >= position) break;
    for (--last; first < last; --last)
      if (T->obj_cent[3 * (size_t)T->ids[last] + axis] < position) break;
    if (first < last) {
      int t = T->ids[first];
      T->ids[first] = T->ids[last];
      T->ids[last] = t;
    } else {
      return first;
    }
  }
}

#define NBINS 16

static Part partition_approx(UTree* T, int node, int b, int e) {
  Part p;
  box_reset(p.bl);
  box_reset(p.br);
  const int n = e - b;
  if (n == 1) {
    p.axis = -1;
    p.split = -1;
    return p;
  }
  if (n == 2) return partition2(T, node, b);
  float cb[6];
  box_reset(cb);
  for (int i = b; i < e; ++i) {
    const float* c = T->obj_cent + 3 * (size_t)T->ids[i];
    for (int k = 0; k < 3; ++k) {
      cb[k] = ref_min(cb[k], c[k]);
      cb[3 + k] = ref_max(cb[3 + k], c[k]);
    }
  }
  const float inv_parent_area = (float)(1.0 / box_area_d(T->bounds + 6 * (size_t)node));
  float best_cost = n * 1.f, best_pos = FLT_MAX;
  int best_axis = -1;
  int bin_count[3][NBINS];
  float bin_box[3][NBINS][6];
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < NBINS; ++i) {
      bin_count[a][i] = 0;
      box_reset(bin_box[a][i]);
    }
  float width[3], scale[3];
  for (int k = 0; k < 3; ++k) {
    width[k] = cb[3 + k] - cb[k];
    scale[k] = (NBINS / width[k]) * .999f;
  }
  /* the reference defines LONGEST_AXIS (as 0), so its #ifdef bins the
     centroid box's longest axis only (DynBVH.cc:39, 2170-2194) */
  const float dxyz[3] = {cb[3] - cb[0], cb[4] - cb[1], cb[5] - cb[2]};
  const int longest = dxyz[0] > dxyz[1] ? (dxyz[0] > dxyz[2] ? 0 : 2)
                                        : (dxyz[1] > dxyz[2] ? 1 : 2);
  for (int i = b; i < e; ++i) {
    const float* ob = T->obj_bounds + 6 * (size_t)T->ids[i];
    const float* c = T->obj_cent + 3 * (size_t)T->ids[i];
    for (int a = longest; a == longest; a++) {
      int w = x86_trunc((c[a] - cb[a]) * scale[a]);
      w = w < 0 ? 0 : w > NBINS - 1 ? NBINS - 1 : w;
      bin_count[a][w]++;
      box_extend(bin_box[a][w], ob);
    }
  }
  for (int a = longest; a == longest; a++) {
    float la[NBINS], ra[NBINS];
    int lc[NBINS], rc[NBINS];
    float lbox[6], rbox[6];
    box_reset(lbox);
    box_reset(rbox);
    int nl = 0, nr = n;
    for (int i = 0; i < NBINS; ++i) {
      nl += bin_count[a][i];
      nr -= bin_count[a][i];
      box_extend(lbox, bin_box[a][i]);
      lc[i] = nl;
      rc[i] = nr;
      la[i] = area_f(lbox);
    }
    for (int i = NBINS - 1; i >= 0; --i) {
      ra[i] = (i == NBINS - 1) ? FLT_MAX : area_f(rbox);
      box_extend(rbox, bin_box[a][i]);
    }
    for (int i = 0; i < NBINS - 1; ++i) {
      const float cost = (la[i] * lc[i] + ra[i] * rc[i]) * inv_parent_area * 1.f + 1.f;
      if (cost < best_cost) {
        best_cost = cost;
        best_axis = a;
        best_pos = cb[a] + width[a] * ((float)(i + 1) / NBINS);
      }
    }
  }
  p.axis = best_axis;
  if (p.axis != -1) {
    int middle = partition_objects(T, b, e, p.axis, best_pos);
    if (middle == b || middle == e) {
      if (n < 3) {
        p.axis = -1;
        p.split = 0;
        return p;
      }
      middle = b + n / 2;
    }
    for (int i = b; i < middle; ++i) box_extend(p.bl, T->obj_bounds + 6 * (size_t)T->ids[i]);
    for (int i = middle; i < e; ++i) box_extend(p.br, T->obj_bounds + 6 * (size_t)T->ids[i]);
    p.split = middle;
    return p;
  }
  p.split = 0;
  return p;
}

static int cmp_int(const void* a, const void* b) {
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* DynBVH::build(nodeID, begin, end, useApproximateBuild = true, exists) */
static void build_approx(UTree* T, int node, int b, int e, int exists) {
  Part p = partition_approx(T, node, b, e);
  if (p.axis == -1) {
    if (exists) return;
    T->child[node] = b;
    T->children[node] = e - b;
    T->axis[node] = 0;
    T->costs[node] = (e - b) * 1.f;
    qsort(T->ids + b, (size_t)(e - b), sizeof(int), cmp_int);
    return;
  }
  const int spot = T->next_free;
  T->next_free += 2;
  if (spot + 2 > T->cap) {
    T->overflow = 1;
    return;
  }
  T->child[node] = spot;
  T->children[node] = 0;
  T->axis[node] = (unsigned char)p.axis;
  box_copy(T->bounds + 6 * (size_t)spot, p.bl);
  box_copy(T->bounds + 6 * (size_t)(spot + 1), p.br);
  build_approx(T, spot, b, p.split, 0);
  if (T->overflow) return;
  build_approx(T, spot + 1, p.split, e, 0);
}

/* ------------------------------------------------------------ rotate --- */

#define NB(i) (T->bounds + 6 * (size_t)(i))

static void guess_axis(UTree* T, int parent, int a, int b) {
  float ov[3];
  for (int k = 0; k < 3; ++k)
    ov[k] = ref_max(NB(a)[k], NB(b)[k]) - ref_min(NB(a)[3 + k], NB(b)[3 + k]);
  const int ax = index_of_max(ov);
  T->axis[parent] = (unsigned char)ax;
  if (NB(a)[3 + ax] > NB(b)[3 + ax]) node_swap(T, a, b);
}

static void rotate_node(UTree* T, int id) {
  const int L = T->child[id], R = L + 1;
  if (T->children[L] > 1) build_approx(T, L, T->child[L], T->child[L] + T->children[L], 1);
  if (T->overflow) return;
  if (T->children[R] > 1) build_approx(T, R, T->child[R], T->child[R] + T->children[R], 1);
  if (T->overflow) return;
  const int LL = T->child[L], LR = LL + 1, RL = T->child[R], RR = RL + 1;
  const int l_leaf = T->children[L] != 0, r_leaf = T->children[R] != 0;
  float* c = T->costs;
  const float node_area = area_f(NB(id));
  const float left_area = area_f(NB(L));
  const float right_area = area_f(NB(R));
  float ll_area = 0.f, lr_area = 0.f, rl_area = 0.f, rr_area = 0.f;
  float box_a[6], box_b[6];
  box_reset(box_a);
  box_reset(box_b);
  float area_a = 0.f, area_b = 0.f;
  int best = 0;
  float best_cost = node_area * 1.f + left_area * c[L] + right_area * c[R];
  if (!l_leaf) {
    ll_area = area_f(NB(LL));
    lr_area = area_f(NB(LR));
    const float partial = node_area * 1.f + right_area * c[R] + lr_area * c[LR] + ll_area * c[LL];
    float b1[6];
    box_copy(b1, NB(R));
    box_extend(b1, NB(LR));
    const float a1 = area_f(b1);
    const float u1 = a1 * 1.f + partial;
    if (u1 < best_cost) {
      best = 1; best_cost = u1; box_copy(box_a, b1); area_a = a1;
    }
    float b2[6];
    box_copy(b2, NB(R));
    box_extend(b2, NB(LL));
    const float a2 = area_f(b2);
    const float u2 = a2 * 1.f + partial;
    if (u2 < best_cost) {
      best = 2; best_cost = u2; box_copy(box_a, b2); area_a = a2;
    }
  }
  if (!r_leaf) {
    rl_area = area_f(NB(RL));
    rr_area = area_f(NB(RR));
    const float partial = node_area * 1.f + left_area * c[L] + rr_area * c[RR] + rl_area * c[RL];
    float b3[6];
    box_copy(b3, NB(L));
    box_extend(b3, NB(RR));
    const float a3 = area_f(b3);
    const float u3 = a3 * 1.f + partial;
    if (u3 < best_cost) {
      best = 3; best_cost = u3; box_copy(box_a, b3); area_a = a3;
    }
    float b4[6];
    box_copy(b4, NB(L));
    box_extend(b4, NB(RL));
    const float a4 = area_f(b4);
    const float u4 = a4 * 1.f + partial;
    if (u4 < best_cost) {
      best = 4; best_cost = u4; box_copy(box_a, b4); area_a = a4;
    }
    if (!l_leaf) {
      const float partial2 = node_area * 1.f + ll_area * c[LL] + lr_area * c[LR] +
                             rl_area * c[RL] + rr_area * c[RR];
      float b5l[6], b5r[6];
      box_copy(b5l, NB(LL));
      box_extend(b5l, NB(RL));
      const float a5l = area_f(b5l);
      box_copy(b5r, NB(LR));
      box_extend(b5r, NB(RR));
      const float a5r = area_f(b5r);
      const float u5 = (a5l + a5r) * 1.f + partial2;
      if (u5 < best_cost) {
        best = 5; best_cost = u5;
        box_copy(box_a, b5l); area_a = a5l;
        box_copy(box_b, b5r); area_b = a5r;
      }
      float b6l[6], b6r[6];
      box_copy(b6l, NB(LL));
      box_extend(b6l, NB(RR));
      const float a6l = area_f(b6l);
      box_copy(b6r, NB(RL));
      box_extend(b6r, NB(LR));
      const float a6r = area_f(b6r);
      const float u6 = (a6l + a6r) * 1.f + partial2;
      if (u6 < best_cost) {
        best = 6; best_cost = u6;
        box_copy(box_a, b6l); area_a = a6l;
        box_copy(box_b, b6r); area_b = a6r;
      }
    }
  }
  c[id] = best_cost / node_area;
  if (best == 0) return;
  const float inv_a = 1 / area_a;
  switch (best) {
    case 1:
      box_copy(NB(L), box_a);
      c[L] = 1.f + ((lr_area * c[LR] + right_area * c[R]) * inv_a);
      node_swap(T, LL, R);
      break;
    case 2:
      box_copy(NB(L), box_a);
      c[L] = 1.f + ((ll_area * c[LL] + right_area * c[R]) * inv_a);
      node_swap(T, LR, R);
      break;
    case 3:
      box_copy(NB(R), box_a);
      c[R] = 1.f + ((rr_area * c[RR] + left_area * c[L]) * inv_a);
      node_swap(T, RL, L);
      break;
    case 4:
      box_copy(NB(R), box_a);
      c[R] = 1.f + ((rl_area * c[RL] + left_area * c[L]) * inv_a);
      node_swap(T, RR, L);
      break;
    case 5:
      box_copy(NB(L), box_a);
      box_copy(NB(R), box_b);
      c[L] = 1.f + ((ll_area * c[LL] + rl_area * c[RL]) * inv_a);
      c[R] = 1.f + ((lr_area * c[LR] + rr_area * c[RR]) / area_b);
      node_swap(T, LR, RL);
      break;
    case 6:
      box_copy(NB(L), box_a);
      box_copy(NB(R), box_b);
      c[L] = 1.f + ((ll_area * c[LL] + rr_area * c[RR]) * inv_a);
      c[R] = 1.f + ((lr_area * c[LR] + rl_area * c[RL]) / area_b);
      node_swap(T, LR, RR);
      break;
  }
  if (best <= 2 || best >= 5) guess_axis(T, L, LL, LR);
  if (best >= 3) guess_axis(T, R, RL, RR);
  guess_axis(T, id, L, R);
}

/* ------------------------------------------------------------ update --- */

static void update_node(UTree* T, int id, int rotate) {
  float* b = NB(id);
  if (T->children[id] != 0) {
    box_reset(b);
    for (int i = 0; i < T->children[id]; ++i)
      box_extend(b, T->obj_bounds + 6 * (size_t)T->ids[T->child[id] + i]);
    T->axis[id] = 0;
    return;
  }
  const int l = T->child[id], r = l + 1;
  update_node(T, l, rotate);
  if (T->overflow) return;
  update_node(T, r, rotate);
  if (T->overflow) return;
  box_reset(b);
  box_extend(b, NB(l));
  box_extend(b, NB(r));
  if (rotate) rotate_node(T, id);
}

static float cost_save(UTree* T, int id) {
  float cost;
  if (T->children[id] != 0) {
    cost = T->children[id] * 1.f;
  } else {
    const int l = T->child[id], r = l + 1;
    const float lc = cost_save(T, l), rc = cost_save(T, r);
    const float area = area_f(NB(id));
    const float la = area_f(NB(l)), ra = area_f(NB(r));
    cost = 1.f + (la * lc + ra * rc) / area;
  }
  T->costs[id] = cost;
  return cost;
}

/* DynBVH::computeCost<true>(0): the per-node costs a rebuild leaves. */
float orq_tree_costs(const float* bounds, const int* child, const int* children, float* costs) {
  UTree T;
  memset(&T, 0, sizeof(T));
  T.bounds = (float*)bounds;
  T.child = (int*)child;
  T.children = (int*)children;
  T.costs = costs;
  return cost_save(&T, 0);
}

/* DynBVH::update(0, 1) after the mesh's vertices moved.  The node arrays
 * have room for cap nodes; *next_free is DynBVH::nextFree.  rotate = 0
 * restates the reference built with TREE_ROT 0 (bounds only).  Returns 0,
 * or 1 when a leaf re-split would need more than cap nodes. */
int orq_tree_update(float* bounds, int* child, int* children, unsigned char* axis,
                    unsigned char* left_cheaper, float* costs, int* ids, int cap,
                    int* next_free, const float* verts, const unsigned* idx, int ntris,
                    int rotate) {
  UTree T;
  T.bounds = bounds;
  T.child = child;
  T.children = children;
  T.axis = axis;
  T.left_cheaper = left_cheaper;
  T.costs = costs;
  T.ids = ids;
  T.cap = cap;
  T.next_free = *next_free;
  T.overflow = 0;
  T.obj_bounds = (float*)malloc(6 * (size_t)(ntris > 0 ? ntris : 1) * sizeof(float));
  T.obj_cent = (float*)malloc(3 * (size_t)(ntris > 0 ? ntris : 1) * sizeof(float));
  if (!T.obj_bounds || !T.obj_cent) {
    free(T.obj_bounds);
    free(T.obj_cent);
    return 2;
  }
  for (int i = 0; i < ntris; ++i) {
    const float* p1 = verts + 3 * (size_t)idx[3 * (size_t)i];
    const float* p2 = verts + 3 * (size_t)idx[3 * (size_t)i + 1];
    const float* p3 = verts + 3 * (size_t)idx[3 * (size_t)i + 2];
    float tb[6] = {p1[0], p1[1], p1[2], p1[0], p1[1], p1[2]};
    for (int k = 0; k < 3; ++k) {
      tb[k] = ref_min(tb[k], p2[k]);
      tb[3 + k] = ref_max(tb[3 + k], p2[k]);
    }
    for (int k = 0; k < 3; ++k) {
      tb[k] = ref_min(tb[k], p3[k]);
      tb[3 + k] = ref_max(tb[3 + k], p3[k]);
    }
    float* ob = T.obj_bounds + 6 * (size_t)i;
    box_reset(ob);
    box_extend(ob, tb);
    for (int k = 0; k < 3; ++k)
      T.obj_cent[3 * (size_t)i + k] = ob[3 + k] * 0.5f + ob[k] * (1 - 0.5f);
  }
  update_node(&T, 0, rotate);
  free(T.obj_bounds);
  free(T.obj_cent);
  *next_free = T.next_free;
  return T.overflow ? 1 : 0;
}
