/*
 * Test infrastructure, not product code: the CPU restatement ("oracle") of
 * Manta's ray-query hot path, used only by tests/, the smoke check and the
 * CPU-baseline leg of bench.py to check the device path.
 *
 * It restates, one ray at a time and in the reference's float operation
 * order (x86-64 SSE scalar float, no FMA contraction: compile with
 * -ffp-contract=off), what the reference computes:
 *
 *   orq_wald_setup    WaldTriangle::setPoints
 *                     (Model/Primitives/WaldTriangle.cc:64-126)
 *   box test          DynBVH::firstIntersects scalar branch
 *                     (Model/Groups/DynBVH.cc:657-681)
 *   traversal order   DynBVH::intersectNode (DynBVH.cc:274-404): closest
 *                     hit visits child (dir[axis] > 0 ? 0 : 1) first, AnyHit
 *                     visits (isLeftCheaper ? 0 : 1) first
 *   Wald test         WaldTriangle::intersect scalar (WaldTriangle.cc:489-555)
 *   KS test           KenslerShirleyTriangle::intersect scalar
 *                     (Model/Primitives/KenslerShirleyTriangle.cc:336-378)
 *   hit acceptance    RayPacket::hit (Interface/RayPacket.h:531-543)
 *   SAH tree cost     DynBVH::computeCost (DynBVH.cc:3389-3416) with
 *                     BBox::computeArea (Core/Geometry/BBox.h:117-121)
 *   camera            PinholeCamera::setup / makeRaysSpecialized scalar
 *                     (Model/Cameras/PinholeCamera.cc:167-198, 356-366) and
 *                     the SingleSampler pixel scale/offset
 *                     (Engine/PixelSamplers/SingleSampler.cc:38-41)
 *   shading           Raytracer::traceRays (Engine/Renderers/Raytracer.cc:49-97),
 *                     Lambertian::shade (Model/Materials/Lambertian.cc:63-246,
 *                     scalar branches), HardShadows::computeShadows
 *                     (Engine/Shadows/HardShadows.cc:46-360, scalar branch),
 *                     PointLight::computeLight (Model/Lights/PointLight.cc:31-79),
 *                     RayPacket normalizeDirections / computeHitPositions /
 *                     computeFFNormals / computeFFGeometricNormals
 *                     (Interface/RayPacket.cc:8-79, 114-146, 205-310).
 *
 * A packet traversal and this per-ray traversal test the same (ray, box) and
 * (ray, triangle) pairs with the same float operations; they can disagree
 * only where two candidate hits tie (which one the traversal order meets
 * first) or where rounding puts a hit within an ulp of a box face.
 * orq_top2 reports the two nearest candidate distances so such rays can be
 * identified.
 *
 * Tree format: the reference DynBVH node array, field by field (DynBVH.h:37-79):
 * bounds[6*i] = min xyz, max xyz; child; children (leaf iff != 0); axis;
 * isLeftCheaper; plus object_ids.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define T_EPSILON 1.e-4f
#define MAXT 1.e19f

typedef struct {
  const float* bounds;
  const int* child;
  const int* children;
  const unsigned char* axis;
  const unsigned char* left_cheaper;
  const int* ids;
  int tri_kind; /* 0 Wald, 1 Kensler-Shirley */
  const float* verts;
  const unsigned* idx;
  const float* wald; /* 12 floats per triangle, see orq_wald_setup */
} Tree;

typedef struct {
  float o[3], d[3], inv[3];
  float minT;
  int hit;  /* reference: hitMatl != 0 */
  int prim;
  float u, v;
  long node_tests, tri_tests;
  int anyhit;
} Ray;

/* ---------------------------------------------------------------- Wald --- */

static float f_abs(float x) { return x < 0.f ? -x : x; }

/* WaldTriangle::setPoints (WaldTriangle.cc:64-126).  Record layout:
 * [n_u, n_v, n_d, k(bits), b_nu, b_nv, b_d, n_k, c_nu, c_nv, c_d, 0]. */
void orq_wald_setup(const float* verts, const unsigned* idx, int ntris,
                    float* rec) {
  for (int t = 0; t < ntris; ++t) {
    const float* p1 = verts + 3 * idx[3 * t + 0];
    const float* p2 = verts + 3 * idx[3 * t + 1];
    const float* p3 = verts + 3 * idx[3 * t + 2];
    float e1[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
    float e2[3] = {p3[0] - p1[0], p3[1] - p1[1], p3[2] - p1[2]};
    float nrm[3] = {e1[1] * e2[2] - e1[2] * e2[1],
                    e1[2] * e2[0] - e1[0] * e2[2],
                    e1[0] * e2[1] - e1[1] * e2[0]};
    /* Vector::normalize (Core/Geometry/Vector.h:322-331) */
    float l = sqrtf(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    float scale = 1 / l;
    nrm[0] *= scale;
    nrm[1] *= scale;
    nrm[2] *= scale;
    unsigned n = 0, u, v;
    if (f_abs(nrm[1]) > f_abs(nrm[n])) n = 1;
    if (f_abs(nrm[2]) > f_abs(nrm[n])) n = 2;
    switch (n) {
      case 0: u = 1; v = 2; break;
      case 1: u = 2; v = 0; break;
      default: u = 0; v = 1; break;
    }
    unsigned k = n;
    float inv_normalk = 1 / nrm[k];
    float n_u = nrm[u] * inv_normalk;
    float n_v = nrm[v] * inv_normalk;
    float n_d = p1[u] * n_u + p1[v] * n_v + p1[k];
    float s;
    float c_nu = +p2[v] - p1[v];
    float c_nv = -p2[u] + p1[u];
    float c_d = -(p1[u] * c_nu + p1[v] * c_nv);
    s = 1.f / (p3[u] * c_nu + p3[v] * c_nv + c_d);
    c_nu *= s;
    c_nv *= s;
    c_d *= s;
    float b_nu = +p3[v] - p1[v];
    float b_nv = -p3[u] + p1[u];
    float b_d = -(p1[u] * b_nu + p1[v] * b_nv);
    s = 1.f / (p2[u] * b_nu + p2[v] * b_nv + b_d);
    b_nu *= s;
    b_nv *= s;
    b_d *= s;
    float* r = rec + 12 * (size_t)t;
    r[0] = n_u;
    r[1] = n_v;
    r[2] = n_d;
    memcpy(&r[3], &k, 4);
    r[4] = b_nu;
    r[5] = b_nv;
    r[6] = b_d;
    r[7] = nrm[k];
    r[8] = c_nu;
    r[9] = c_nv;
    r[10] = c_d;
    r[11] = 0.f;
  }
}

/* RayPacket::hit (RayPacket.h:531-543). */
static int ray_hit(Ray* r, float t, int prim) {
  if (t > T_EPSILON && t < r->minT) {
    r->minT = t;
    r->hit = 1;
    r->prim = prim;
    return 1;
  }
  return 0;
}

/* WaldTriangle::intersect scalar (WaldTriangle.cc:489-555), one ray. */
static void wald_test(const Tree* T, int tri, Ray* r) {
  const float* w = T->wald + 12 * (size_t)tri;
  unsigned k;
  memcpy(&k, &w[3], 4);
  const int axis = (int)k;
  const int ku = (k == 2) ? 0 : (int)k + 1;
  const int kv = (k == 0) ? 2 : (int)k - 1;
  const float n_u = w[0], n_v = w[1], n_d = w[2];
  const float nd0 = n_u * r->d[ku] + n_v * r->d[kv] + r->d[axis];
  const float nd = 1.f / nd0;
  const float org_k = r->o[axis], org_ku = r->o[ku], org_kv = r->o[kv];
  const float f0 = n_d - (org_k + n_u * org_ku + n_v * org_kv);
  const float f = f0 * nd;
  if (f < T_EPSILON || f > r->minT) return;
  const float hu = org_ku + f * r->d[ku];
  const float hv = org_kv + f * r->d[kv];
  const float lambda = w[6] + hu * w[4] + hv * w[5];
  if (lambda < 0.f) return;
  const float mue = w[10] + hu * w[8] + hv * w[9];
  if (mue < 0.f || mue + lambda > 1.f) return;
  if (ray_hit(r, f, tri)) {
    r->u = lambda;
    r->v = mue;
  }
}

/* KenslerShirleyTriangle::intersect scalar (KenslerShirleyTriangle.cc:336-378). */
static void ks_test(const Tree* T, int tri, Ray* r) {
  const float* p0 = T->verts + 3 * T->idx[3 * tri + 0];
  const float* p1 = T->verts + 3 * T->idx[3 * tri + 1];
  const float* p2 = T->verts + 3 * T->idx[3 * tri + 2];
  const float e0[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
  const float e1[3] = {p0[0] - p2[0], p0[1] - p2[1], p0[2] - p2[2]};
  const float n[3] = {e0[1] * e1[2] - e0[2] * e1[1],
                      e0[2] * e1[0] - e0[0] * e1[2],
                      e0[0] * e1[1] - e0[1] * e1[0]};
  const float oldt = r->minT;
  const float rcp = 1.0f / (n[0] * r->d[0] + n[1] * r->d[1] + n[2] * r->d[2]);
  const float e2[3] = {p0[0] - r->o[0], p0[1] - r->o[1], p0[2] - r->o[2]};
  const float toverd = (n[0] * e2[0] + n[1] * e2[1] + n[2] * e2[2]) * rcp;
  if (toverd > oldt - T_EPSILON || toverd < T_EPSILON) return;
  const float im[3] = {e2[1] * r->d[2] - e2[2] * r->d[1],
                       e2[2] * r->d[0] - e2[0] * r->d[2],
                       e2[0] * r->d[1] - e2[1] * r->d[0]};
  const float uoverd = (im[0] * e1[0] + im[1] * e1[1] + im[2] * e1[2]) * rcp;
  if (uoverd < 0.0f) return;
  const float voverd = (im[0] * e0[0] + im[1] * e0[1] + im[2] * e0[2]) * rcp;
  if (uoverd + voverd > 1.0f || voverd < 0.0f) return;
  if (ray_hit(r, toverd, tri)) {
    r->u = uoverd;
    r->v = voverd;
  }
}

/* DynBVH::firstIntersects scalar box test (DynBVH.cc:666-681). */
static int box_test(const float* b, const Ray* r) {
  float tmin = T_EPSILON;
  float tmax = r->minT;
  for (int c = 0; c < 3; c++) {
    float t0 = (b[c] - r->o[c]) * r->inv[c];
    float t1 = (b[3 + c] - r->o[c]) * r->inv[c];
    float near = (t0 < t1) ? t0 : t1;
    float far = (t0 < t1) ? t1 : t0;
    tmin = (tmin < near) ? near : tmin;
    tmax = (far < tmax) ? far : tmax;
  }
  return tmin <= tmax;
}

/* DynBVH::intersectNode (DynBVH.cc:274-404) for one ray. */
static void visit(const Tree* T, int node, Ray* r) {
  if (r->anyhit && r->hit) return; /* firstIntersects skips hit rays */
  r->node_tests++;
  if (!box_test(T->bounds + 6 * (size_t)node, r)) return;
  const int nch = T->children[node];
  const int first = T->child[node];
  if (nch != 0) {
    for (int i = 0; i < nch; ++i) {
      const int obj = T->ids[first + i];
      r->tri_tests++;
      if (T->tri_kind == 0)
        wald_test(T, obj, r);
      else
        ks_test(T, obj, r);
      if (r->anyhit && r->hit) {
        /* OpaqueShadower terminates the ray (DynBVH.cc:331-349) */
        r->minT = T_EPSILON;
        return;
      }
    }
    return;
  }
  int front;
  if (r->anyhit)
    front = T->left_cheaper[node] ? 0 : 1;
  else
    front = r->d[T->axis[node]] > 0 ? 0 : 1;
  visit(T, first + front, r);
  visit(T, first + 1 - front, r);
}

static void ray_init(Ray* r, const float* org, const float* dir, int n, int i,
                     float tmax, int anyhit) {
  for (int c = 0; c < 3; ++c) {
    r->o[c] = org[c * n + i];
    r->d[c] = dir[c * n + i];
    /* RayPacket::actualComputeInverseDirections (RayPacket.cc:106-110) */
    r->inv[c] = (float)1 / r->d[c];
  }
  r->minT = tmax;
  r->hit = 0;
  r->prim = -1;
  r->u = r->v = 0.f;
  r->node_tests = r->tri_tests = 0;
  r->anyhit = anyhit;
}

/* Closest-hit / any-hit query of n rays (SoA org/dir).  Outputs hit flag,
 * t (minT after the query), triangle id, u, v; optional per-ray node and
 * triangle test counts. */
int orq_trace(const float* bounds, const int* child, const int* children,
              const unsigned char* axis, const unsigned char* left_cheaper,
              const int* ids, int tri_kind, const float* verts,
              const unsigned* idx, const float* wald, int n, const float* org,
              const float* dir, const float* tmax, int anyhit, int* hit,
              float* t, int* prim, float* u, float* v, int* node_tests,
              int* tri_tests) {
  Tree T = {bounds, child, children, axis, left_cheaper, ids,
            tri_kind, verts, idx, wald};
  for (int i = 0; i < n; ++i) {
    Ray r;
    ray_init(&r, org, dir, n, i, tmax[i], anyhit);
    visit(&T, 0, &r);
    hit[i] = r.hit;
    t[i] = r.minT;
    prim[i] = r.hit ? r.prim : -1;
    u[i] = r.u;
    v[i] = r.v;
    if (node_tests) node_tests[i] = (int)r.node_tests;
    if (tri_tests) tri_tests[i] = (int)r.tri_tests;
  }
  return 0;
}

/* -------------------------------------------------- near-tie detection --- */

typedef struct {
  float t1, t2;
  int p1, p2;
} Top2;

static void top2_visit(const Tree* T, int node, Ray* r, Top2* k) {
  /* cull against the second-nearest candidate */
  r->minT = k->t2;
  if (!box_test(T->bounds + 6 * (size_t)node, r)) return;
  const int nch = T->children[node];
  const int first = T->child[node];
  if (nch != 0) {
    for (int i = 0; i < nch; ++i) {
      const int obj = T->ids[first + i];
      r->minT = k->t2;
      r->hit = 0;
      if (T->tri_kind == 0)
        wald_test(T, obj, r);
      else
        ks_test(T, obj, r);
      if (r->hit) {
        float tt = r->minT;
        if (tt < k->t1) {
          k->t2 = k->t1;
          k->p2 = k->p1;
          k->t1 = tt;
          k->p1 = obj;
        } else {
          k->t2 = tt;
          k->p2 = obj;
        }
      }
    }
    return;
  }
  top2_visit(T, first, r, k);
  top2_visit(T, first + 1, r, k);
}

/* Nearest and second-nearest candidate hit distance per ray (MAXT/tmax when
 * absent) over all triangles the ray hits in (T_EPSILON, tmax). */
int orq_top2(const float* bounds, const int* child, const int* children,
             const unsigned char* axis, const unsigned char* left_cheaper,
             const int* ids, int tri_kind, const float* verts,
             const unsigned* idx, const float* wald, int n, const float* org,
             const float* dir, const float* tmax, float* t1, float* t2,
             int* p1, int* p2) {
  Tree T = {bounds, child, children, axis, left_cheaper, ids,
            tri_kind, verts, idx, wald};
  for (int i = 0; i < n; ++i) {
    Ray r;
    ray_init(&r, org, dir, n, i, tmax[i], 0);
    Top2 k = {tmax[i], tmax[i], -1, -1};
    top2_visit(&T, 0, &r, &k);
    t1[i] = k.t1;
    t2[i] = k.t2;
    p1[i] = k.p1;
    p2[i] = k.p2;
  }
  return 0;
}

/* ---------------------------------------------------------- SAH cost --- */

static float box_area(const float* b) {
  /* BBox::computeArea: 2 * (dx*dy + dy*dz + dx*dz) in float */
  float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
  return 2 * (dx * dy + dy * dz + dx * dz);
}

static float cost_rec(const float* bounds, const int* child,
                      const int* children, int node) {
  if (children[node] != 0) return children[node] * 1.f;
  const int l = child[node], r = child[node] + 1;
  float lc = cost_rec(bounds, child, children, l);
  float rc = cost_rec(bounds, child, children, r);
  float area = box_area(bounds + 6 * (size_t)node);
  float la = box_area(bounds + 6 * (size_t)l);
  float ra = box_area(bounds + 6 * (size_t)r);
  return 1.f + (la * lc + ra * rc) / area;
}

/* DynBVH::computeCost<>(0) (DynBVH.cc:3389-3416), C_isec = C_trav = 1. */
double orq_sah_cost(const float* bounds, const int* child, const int* children) {
  return cost_rec(bounds, child, children, 0);
}

/* ------------------------------------------------------------ camera --- */

static void v_normalize(float* a) {
  float l = sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  float s = 1 / l;
  a[0] *= s;
  a[1] *= s;
  a[2] *= s;
}

static void v_cross(const float* a, const float* b, float* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

/* -------------------------------------------- ambient and background --- */

/* A frame's ambient light and background beyond the constant forms:
 * ambient_kind 1 = EyeAmbient, background_kind 1 = LinearBackground with
 * cup = the frame's background colour, cdown = down, and up as given (the
 * constructor normalises it).  NULL or zero kinds = ConstantAmbient /
 * ConstantBackground. */
typedef struct {
  int ambient_kind;
  int background_kind;
  float down[3];
  float up[3];
} orq_env;

/* Vector Dot (Core/Geometry/VectorT.h:443-449): result = 0, then += a[i]b[i]. */
static float v_dot(const float* a, const float* b) {
  float r = 0;
  for (int i = 0; i < 3; ++i) r += a[i] * b[i];
  return r;
}

/* EyeAmbient::computeAmbient (Model/AmbientLights/EyeAmbient.cc:29-44):
 * cos_theta = -Dot(eyeDir, ffnormal) * (1 - minLighting) + minLighting with
 * minLighting 0.5, ambient = colour * cos_theta; ConstantAmbient copies the
 * colour. */
static void env_ambient(const orq_env* E, const float* color, const float* d,
                        const float* ffn, float* out) {
  if (E && E->ambient_kind == 1) {
    const float min_lighting = 0.5f;
    const float cos_theta = -v_dot(d, ffn) * (1 - min_lighting) + min_lighting;
    for (int c = 0; c < 3; ++c) out[c] = color[c] * cos_theta;
  } else {
    for (int c = 0; c < 3; ++c) out[c] = color[c];
  }
}

/* LinearBackground (Model/Backgrounds/LinearBackground.cc:15-40): the
 * constructor's up.normalize() (VectorT::normalize, VectorT.h:324-333), then
 * t = 0.5 * (1 + Dot(d, up)) and colour = cup * t + cdown * (1 - t);
 * ConstantBackground returns cup. */
static void env_background(const orq_env* E, const float* cup, const float* d, float* out) {
  if (E && E->background_kind == 1) {
    float up[3] = {E->up[0], E->up[1], E->up[2]};
    float sum = 0;
    for (int i = 0; i < 3; ++i) sum += up[i] * up[i];
    const float l = sqrtf(sum);
    const float scale = 1 / l;
    for (int i = 0; i < 3; ++i) up[i] *= scale;
    const float t = 0.5f * (1 + v_dot(d, up));
    for (int c = 0; c < 3; ++c) out[c] = cup[c] * t + E->down[c] * (1 - t);
  } else {
    for (int c = 0; c < 3; ++c) out[c] = cup[c];
  }
}

/* PinholeCamera::setup (PinholeCamera.cc:167-198): out = eye, direction, u, v. */
void orq_camera_basis(const float* eye, const float* lookat, const float* up_in,
                      float hfov, float vfov, float* out12) {
  float dir[3] = {lookat[0] - eye[0], lookat[1] - eye[1], lookat[2] - eye[2]};
  float nearZ = sqrtf(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  float up[3] = {up_in[0], up_in[1], up_in[2]};
  v_normalize(up);
  float v[3], u[3];
  v_cross(dir, up, v);
  v_normalize(v);
  v_cross(v, dir, u);
  v_normalize(u);
  const double pi = 3.14159265358979323846;
  float height = (float)(nearZ * tan((0.5 * vfov) * (pi / 180.)));
  u[0] *= height;
  u[1] *= height;
  u[2] *= height;
  float width = (float)(nearZ * tan((0.5 * hfov) * (pi / 180.)));
  v[0] *= width;
  v[1] *= width;
  v[2] *= width;
  for (int i = 0; i < 3; ++i) {
    out12[i] = eye[i];
    out12[3 + i] = dir[i];
    out12[6 + i] = u[i];
    out12[9 + i] = v[i];
  }
}

/* SingleSampler scale/offset + PinholeCamera::makeRaysSpecialized<true,false>
 * scalar branch: o = eye, d = normalize(v*px + u*py + direction). */
static void primary_ray(const float* cam, int xres, int yres, int x, int y,
                        float* o, float* d) {
  const float xscale = (float)2 / xres;
  const float yscale = (float)2 / yres;
  const float xoffset = (-xres / (float)2 + (float)0.5) * xscale;
  const float yoffset = (-yres / (float)2 + (float)0.5) * yscale;
  const float px = (float)x * xscale + xoffset;
  const float py = (float)y * yscale + yoffset;
  const float* dir = cam + 3;
  const float* u = cam + 6;
  const float* v = cam + 9;
  for (int c = 0; c < 3; ++c) {
    o[c] = cam[c];
    d[c] = v[c] * px + u[c] * py + dir[c];
  }
  v_normalize(d);
}

/* Primary rays of an xres x yres frame, SoA. */
void orq_primary_rays(const float* cam, int xres, int yres, float* org,
                      float* dir) {
  const int n = xres * yres;
  for (int y = 0; y < yres; ++y)
    for (int x = 0; x < xres; ++x) {
      float o[3], d[3];
      primary_ray(cam, xres, yres, x, y, o, d);
      const int i = y * xres + x;
      for (int c = 0; c < 3; ++c) {
        org[c * n + i] = o[c];
        dir[c * n + i] = d[c];
      }
    }
}

/* Unit geometric normal of triangle `tri`: WaldTriangle::computeNormal
 * without vertex normals (WaldTriangle.cc:578-590) or the normalised
 * KenslerShirleyTriangle::computeNormal cross product
 * (KenslerShirleyTriangle.cc:396-405, normalised by RayPacket.cc:177-186). */
static void tri_normal(const Tree* T, int tri, float* nrm) {
  if (T->tri_kind == 0) {
    const float* w = T->wald + 12 * (size_t)tri;
    unsigned k;
    memcpy(&k, &w[3], 4);
    const int ku = (k == 2) ? 0 : (int)k + 1;
    const int kv = (k == 0) ? 2 : (int)k - 1;
    const float n_k = w[7];
    nrm[k] = n_k;
    nrm[ku] = n_k * w[0];
    nrm[kv] = n_k * w[1];
  } else {
    const float* p0 = T->verts + 3 * T->idx[3 * tri + 0];
    const float* p1 = T->verts + 3 * T->idx[3 * tri + 1];
    const float* p2 = T->verts + 3 * T->idx[3 * tri + 2];
    const float e0[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const float e1[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    v_cross(e0, e1, nrm);
    float sum = 0;
    for (int j = 0; j < 3; ++j) sum += nrm[j] * nrm[j];
    float scale = 1 / sqrtf(sum);
    for (int j = 0; j < 3; ++j) nrm[j] *= scale;
  }
}

/* Whitted frame: Raytracer + Lambertian + HardShadows(point lights).
 * lights: nl x (pos xyz, rgb).  mat_rgb/face_mat: diffuse colour per
 * material.  Outputs rgb (3 per pixel), primary t and triangle id, the
 * number of shadow rays sent, optional per-pixel occlusion bits (bit j set =
 * light j unshadowed) and optional traversal counts: counts[0..3] = node
 * tests and triangle tests of the primary rays, then of the shadow rays. */
long long orq_render_whitted(const float* bounds, const int* child,
                             const int* children, const unsigned char* axis,
                             const unsigned char* left_cheaper, const int* ids,
                             int tri_kind, const float* verts,
                             const unsigned* idx, const float* wald,
                             const unsigned* face_mat, const float* mat_rgb,
                             const float* cam, int xres, int yres,
                             const float* lights, int nl, const float* ambient,
                             const float* background, int y0, int y1,
                             float* rgb, float* tprim, int* prim,
                             int* lit_bits, long long* counts, const orq_env* env) {
  Tree T = {bounds, child, children, axis, left_cheaper, ids,
            tri_kind, verts, idx, wald};
  long long shadow_rays = 0;
  for (int y = y0; y < y1; ++y) {
    for (int x = 0; x < xres; ++x) {
      const size_t pix = (size_t)y * xres + x;
      Ray r;
      primary_ray(cam, xres, yres, x, y, r.o, r.d);
      for (int c = 0; c < 3; ++c) r.inv[c] = (float)1 / r.d[c];
      r.minT = MAXT;
      r.hit = 0;
      r.prim = -1;
      r.u = r.v = 0.f;
      r.anyhit = 0;
      r.node_tests = r.tri_tests = 0;
      visit(&T, 0, &r);
      if (counts) {
        counts[0] += r.node_tests;
        counts[1] += r.tri_tests;
      }
      tprim[pix] = r.minT;
      prim[pix] = r.hit ? r.prim : -1;
      if (lit_bits) lit_bits[pix] = 0;
      if (!r.hit) {
        /* Background::shade */
        env_background(env, background, r.d, rgb + 3 * pix);
        continue;
      }
      /* Lambertian::shade.  Directions are already unit length
       * (NormalizedDirections set by the camera), so normalizeDirections is
       * a no-op here. */
      const float* kd = mat_rgb + 3 * face_mat[r.prim];
      float nrm[3];
      tri_normal(&T, r.prim, nrm);
      float ffn[3];
      const float dn = nrm[0] * r.d[0] + nrm[1] * r.d[1] + nrm[2] * r.d[2];
      for (int c = 0; c < 3; ++c) ffn[c] = (dn <= 0) ? nrm[c] : -nrm[c];
      /* geometric normal == shading normal for both triangle kinds here */
      const float* ffg = ffn;
      float total[3];
      env_ambient(env, ambient, r.d, ffn, total);
      float hp[3];
      for (int c = 0; c < 3; ++c) hp[c] = r.o[c] + r.d[c] * r.minT;
      for (int j = 0; j < nl; ++j) {
        const float* L = lights + 6 * j;
        float sd[3] = {L[0] - hp[0], L[1] - hp[1], L[2] - hp[2]};
        if (!(sd[0] * ffg[0] + sd[1] * ffg[1] + sd[2] * ffg[2] > 0))
          continue; /* masked: counts as shadowed */
        Ray s;
        for (int c = 0; c < 3; ++c) {
          s.o[c] = hp[c];
          s.d[c] = sd[c];
          s.inv[c] = (float)1 / sd[c];
        }
        s.minT = 1 - T_EPSILON;
        s.hit = 0;
        s.prim = -1;
        s.u = s.v = 0.f;
        s.anyhit = 1;
        s.node_tests = s.tri_tests = 0;
        shadow_rays++;
        visit(&T, 0, &s);
        if (counts) {
          counts[2] += s.node_tests;
          counts[3] += s.tri_tests;
        }
        if (s.hit) continue;
        if (lit_bits) lit_bits[pix] |= 1 << j;
        /* shadowRays.normalizeDirections (RayPacket.cc:61-71) */
        float sum = 0;
        for (int c = 0; c < 3; ++c) sum += sd[c] * sd[c];
        float length = sqrtf(sum);
        float scale = 1 / length;
        for (int c = 0; c < 3; ++c) sd[c] *= scale;
        const float cos_theta = sd[0] * ffn[0] + sd[1] * ffn[1] + sd[2] * ffn[2];
        for (int c = 0; c < 3; ++c) total[c] += L[3 + c] * cos_theta;
      }
      for (int c = 0; c < 3; ++c) rgb[3 * pix + c] = total[c] * kd[c];
    }
  }
  return shadow_rays;
}

/* ------------------------------------------------------ path tracing --- */
/* Restatement of the device path-tracing wavefront (rfmanta_b200/csrc/
 * rq_path.cu), which follows KajiyaPathtracer::traceEyeRays
 * (Engine/Renderers/KajiyaPathtracer.cc:113-302), Lambertian::sampleBSDF
 * (Model/Materials/Lambertian.cc:248-280), AreaLight::computeLight
 * (Model/Lights/AreaLight.cc:25-54) with Parallelogram::getRandomPoints
 * (Model/Primitives/Parallelogram.cc:569-614), HardShadows' cull and
 * russian_roulette_full (KajiyaPathtracer.cc:389-478), one path at a time.
 * Random numbers: PCG32 (O'Neill 2014); sin/cos: quadrant reduction of
 * 2*pi*u plus Taylor polynomials, evaluated with the same separately
 * rounded float operations as the device. */

typedef struct {
  uint64_t state, inc;
} Pcg32;

static uint32_t pcg_next(Pcg32* g) {
  uint64_t old = g->state;
  g->state = old * 6364136223846793005ULL + g->inc;
  uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  uint32_t rot = (uint32_t)(old >> 59u);
  return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

static void pcg_seed(Pcg32* g, uint64_t initstate, uint64_t initseq) {
  g->state = 0u;
  g->inc = (initseq << 1u) | 1u;
  pcg_next(g);
  g->state += initstate;
  pcg_next(g);
}

static float pcg_float(Pcg32* g) {
  return (float)(pcg_next(g) >> 8) * (1.0f / 16777216.0f);
}

static void sincos_2pi(float u, float* c, float* s) {
  const float u4 = u * 4.f;
  const float qf = floorf(u4);
  const int q = (int)qf & 3;
  const float f = u4 - qf;
  const float y = f * 1.57079632679489662f;
  const float y2 = y * y;
  float ps = 1.f - y2 * (1.f / 110.f);
  ps = 1.f - (y2 * (1.f / 72.f)) * ps;
  ps = 1.f - (y2 * (1.f / 42.f)) * ps;
  ps = 1.f - (y2 * (1.f / 20.f)) * ps;
  ps = 1.f - (y2 * (1.f / 6.f)) * ps;
  const float sy = y * ps;
  float pc = 1.f - y2 * (1.f / 132.f);
  pc = 1.f - (y2 * (1.f / 90.f)) * pc;
  pc = 1.f - (y2 * (1.f / 56.f)) * pc;
  pc = 1.f - (y2 * (1.f / 30.f)) * pc;
  pc = 1.f - (y2 * (1.f / 12.f)) * pc;
  const float cy = 1.f - (y2 * 0.5f) * pc;
  switch (q) {
    case 0: *c = cy; *s = sy; break;
    case 1: *c = -sy; *s = cy; break;
    case 2: *c = -cy; *s = -sy; break;
    default: *c = sy; *s = -cy; break;
  }
}

void orq_sincos_2pi(const float* u, int n, float* c, float* s) {
  for (int i = 0; i < n; ++i) sincos_2pi(u[i], &c[i], &s[i]);
}

/* params (float): cam[12], light_anchor[3], light_v1[3], light_v2[3],
 * light_color[3], background[3], ambient[3]; iparams: xres, yres, spp, max_depth,
 * rr_depth.  Writes rgb per pixel, ray counts[2] (extension, shadow), and
 * optionally prim[max_depth][n_paths] (-2 where a path had ended). */
void orq_render_path(const float* bounds, const int* child, const int* children,
                     const unsigned char* axis, const unsigned char* left_cheaper,
                     const int* ids, int tri_kind, const float* verts,
                     const unsigned* idx, const float* wald, const unsigned* face_mat,
                     const float* mat_rgb, const float* fp, const int* ip,
                     unsigned long long seed, long long p0, long long p1, float* rad_out,
                     long long* counts, int* dbg_prim, const orq_env* env) {
  Tree T = {bounds, child, children, axis, left_cheaper, ids,
            tri_kind, verts, idx, wald};
  const float* cam = fp;
  const float* la = fp + 12;
  const float* lv1 = fp + 15;
  const float* lv2 = fp + 18;
  const float* lcol = fp + 21;
  const float* bg = fp + 24;
  const float* amb = fp + 27;
  const int xres = ip[0], yres = ip[1], spp = ip[2], maxd = ip[3], rrd = ip[4];
  int strata = 1;
  while (strata * strata < spp) ++strata;
  const long long npaths = (long long)xres * yres * spp;
  /* Parallelogram (Parallelogram.cc:26-35) */
  float ln[3];
  v_cross(lv1, lv2, ln);
  const float ll = sqrtf(ln[0] * ln[0] + ln[1] * ln[1] + ln[2] * ln[2]);
  const float lsc = 1 / ll;
  for (int c = 0; c < 3; ++c) ln[c] = ln[c] * lsc;
  const float inv_area = (float)1 / ll;
  const float xscale = 2.f / (float)xres, yscale = 2.f / (float)yres;
  const float xo = ((float)(-xres) / 2.f) * xscale, yo = ((float)(-yres) / 2.f) * yscale;
  for (long long g = p0; g < p1; ++g) {
    Pcg32 rng;
    pcg_seed(&rng, seed ^ ((unsigned long long)g * 0x9E3779B97F4A7C15ULL),
             (unsigned long long)g);
    const long long pix = g / spp;
    const int s = (int)(g - pix * spp);
    const int x = (int)(pix % xres), y = (int)(pix / xres);
    float jx = 0.5f, jy = 0.5f;
    if (spp > 1) {
      const int sx = s % strata, sy = s / strata;
      jx = ((float)sx + pcg_float(&rng)) / (float)strata;
      jy = ((float)sy + pcg_float(&rng)) / (float)strata;
    }
    const float px = ((float)x + jx) * xscale + xo;
    const float py = ((float)y + jy) * yscale + yo;
    Ray r;
    float d[3];
    for (int c = 0; c < 3; ++c) {
      r.o[c] = cam[c];
      d[c] = cam[9 + c] * px + cam[6 + c] * py + cam[3 + c];
    }
    v_normalize(d);
    for (int c = 0; c < 3; ++c) r.d[c] = d[c];
    float imp[3] = {1.f, 1.f, 1.f}, rad[3] = {0.f, 0.f, 0.f};
    for (int depth = 0; depth < maxd; ++depth) {
      for (int c = 0; c < 3; ++c) r.inv[c] = (float)1 / r.d[c];
      r.minT = MAXT;
      r.hit = 0;
      r.prim = -1;
      r.anyhit = 0;
      visit(&T, 0, &r);
      counts[0]++;
      if (dbg_prim) dbg_prim[(size_t)depth * npaths + g] = r.hit ? r.prim : -1;
      if (!r.hit) {
        float bgc[3];
        env_background(env, bg, r.d, bgc);
        for (int c = 0; c < 3; ++c) rad[c] = rad[c] + bgc[c] * imp[c];
        break;
      }
      float hp[3], ng[3], ffn[3];
      for (int c = 0; c < 3; ++c) hp[c] = r.o[c] + r.d[c] * r.minT;
      tri_normal(&T, r.prim, ng);
      const float dn = ng[0] * r.d[0] + ng[1] * r.d[1] + ng[2] * r.d[2];
      for (int c = 0; c < 3; ++c) ffn[c] = (dn <= 0.f) ? ng[c] : -ng[c];
      const float r1 = pcg_float(&rng);
      const float r2 = pcg_float(&rng);
      const float sintheta = sqrtf(r1);
      const float costheta = sqrtf(1.f - r1);
      float cph, sph;
      sincos_2pi(r2, &cph, &sph);
      const float cosphi = cph * sintheta;
      const float sinphi = sph * sintheta;
      float v1[3];
      {
        const float d2 = ffn[2] * ffn[2];
        const float d1 = ffn[1] * ffn[1];
        if (d2 + d1 < 1e-4f) {
          v1[0] = -ffn[2];
          v1[1] = 0.f;
          v1[2] = ffn[0];
        } else {
          v1[0] = 0.f;
          v1[1] = ffn[2];
          v1[2] = -ffn[1];
        }
        v_normalize(v1);
      }
      float v2[3];
      v_cross(v1, ffn, v2);
      float nd[3];
      for (int c = 0; c < 3; ++c) nd[c] = ffn[c] * costheta + v1[c] * cosphi + v2[c] * sinphi;
      const float* kd = mat_rgb + 3 * face_mat[r.prim];
      for (int c = 0; c < 3; ++c) imp[c] = imp[c] * kd[c];
      /* do_ambient_on_maxdepth (KajiyaPathtracer.cc:259-279): ambient * kd
         times the importance (which holds this kd) where the path reaches
         its last bounce */
      if (depth + 1 >= maxd) {
        /* By then sampleBSDF has written nd into the packet, and
           Lambertian::shade recomputes the face-forward normals against it
           (RayPacket::computeFFNormals, RayPacket.cc:205-233; the flag
           sampleBSDF set lived in a sub-packet), which EyeAmbient reads. */
        float fn[3], a[3];
        const float dd = ng[0] * nd[0] + ng[1] * nd[1] + ng[2] * nd[2];
        for (int c = 0; c < 3; ++c) fn[c] = (dd <= 0.f) ? ng[c] : -ng[c];
        env_ambient(env, amb, nd, fn, a);
        for (int c = 0; c < 3; ++c) rad[c] = rad[c] + (a[c] * kd[c]) * imp[c];
      }
      const float lr1 = pcg_float(&rng);
      const float lr2 = pcg_float(&rng);
      float ld[3];
      for (int c = 0; c < 3; ++c) ld[c] = (la[c] + lr1 * lv1[c] + lr2 * lv2[c]) - hp[c];
      const float len = sqrtf(ld[0] * ld[0] + ld[1] * ld[1] + ld[2] * ld[2]);
      {
        const float sc = 1.f / len;
        for (int c = 0; c < 3; ++c) ld[c] = ld[c] * sc;
      }
      const float cosine = -(ld[0] * ln[0] + ld[1] * ln[1] + ld[2] * ln[2]);
      if (cosine > 0.f && ld[0] * ffn[0] + ld[1] * ffn[1] + ld[2] * ffn[2] > 0.f) {
        Ray sr;
        for (int c = 0; c < 3; ++c) {
          sr.o[c] = hp[c];
          sr.d[c] = ld[c];
          sr.inv[c] = (float)1 / ld[c];
        }
        sr.minT = len - T_EPSILON;
        sr.hit = 0;
        sr.prim = -1;
        sr.anyhit = 1;
        counts[1]++;
        visit(&T, 0, &sr);
        if (!sr.hit) {
          const float solid_pdf = inv_area * (len * len);
          const float f = cosine / solid_pdf;
          const float sum = ld[0] * ld[0] + ld[1] * ld[1] + ld[2] * ld[2];
          const float sc = 1.f / sqrtf(sum);
          float ldn[3];
          for (int c = 0; c < 3; ++c) ldn[c] = ld[c] * sc;
          const float w = ffn[0] * ldn[0] + ffn[1] * ldn[1] + ffn[2] * ldn[2];
          for (int c = 0; c < 3; ++c) rad[c] = rad[c] + (imp[c] * (f * lcol[c])) * w;
        }
      }
      if (depth + 1 >= maxd) break;
      if (depth >= rrd && depth != maxd - 1) {
        /* russian_roulette_full (KajiyaPathtracer.cc:389-478): killed when
           rr > max(reflectance); the reference's 1/max scale loop runs over
           the killed rays past newEnd (468-475), so survivors keep their
           importance unscaled */
        const float rr = pcg_float(&rng);
        const float mx = fmaxf(fmaxf(kd[0], kd[1]), kd[2]);
        if (rr > mx) break;
      }
      for (int c = 0; c < 3; ++c) {
        r.o[c] = hp[c];
        r.d[c] = nd[c];
      }
    }
    for (int c = 0; c < 3; ++c) rad_out[3 * (g - p0) + c] = rad[c];
  }
}

/* ------------------------------------------------- two-level scenes --- */
/* Scenes given as a "world": a flat triangle tree, or a top-level tree whose
 * objects are instances of inner triangle trees.  Instance kinds:
 *   0  InstanceT (Model/Instances/InstanceT.cc:60-90): the ray enters with
 *      o - translation, the same direction and the current minT; a closer
 *      inner hit is accepted through RayPacket::hit.  In an AnyHit query the
 *      inner DynBVH pins an occluded ray's minT to T_EPSILON (DynBVH.cc:
 *      331-349) and RayPacket::hit(T_EPSILON) fails, so the top level never
 *      sees that occlusion: any-hit queries skip these instances.
 *   1  the inner DynBVH as an object of the top-level group itself
 *      (translation 0): hits and occlusion as for its own triangles. */

typedef struct {
  const float* bounds;
  const int* child;
  const int* children;
  const unsigned char* axis;
  const unsigned char* left_cheaper;
  const int* ids;
  int tri_kind;
  const float* verts;
  const unsigned* idx;
  const float* wald;
  const unsigned* face_mat;
} orq_tree;

typedef struct {
  const orq_tree* top;   /* flat world: the triangle tree */
  const orq_tree* inner; /* NULL for a flat world */
  const int* inst_scene;
  const float* inst_T;
  const int* inst_kind;
} orq_world;

static Tree as_tree(const orq_tree* t) {
  Tree T = {t->bounds, t->child, t->children, t->axis, t->left_cheaper,
            t->ids, t->tri_kind, t->verts, t->idx, t->wald};
  return T;
}

/* DynBVH::intersectNode of the top-level tree; leaves hand the ray to the
 * instances. */
static void visit_top(const orq_world* W, int node, Ray* r, int* inst) {
  const orq_tree* T = W->top;
  if (r->anyhit && r->hit) return;
  r->node_tests++;
  if (!box_test(T->bounds + 6 * (size_t)node, r)) return;
  const int nch = T->children[node];
  const int first = T->child[node];
  if (nch != 0) {
    for (int i = 0; i < nch; ++i) {
      const int k = T->ids[first + i];
      const int kind = W->inst_kind ? W->inst_kind[k] : 0;
      if (r->anyhit && kind == 0) continue;
      const Tree IT = as_tree(&W->inner[W->inst_scene[k]]);
      Ray lr = *r;
      for (int c = 0; c < 3; ++c) lr.o[c] = r->o[c] - W->inst_T[3 * k + c];
      lr.hit = 0;
      lr.prim = -1;
      lr.u = lr.v = 0.f;
      visit(&IT, 0, &lr);
      r->node_tests = lr.node_tests;
      r->tri_tests = lr.tri_tests;
      if (lr.hit) {
        r->minT = lr.minT;
        r->hit = 1;
        r->prim = lr.prim;
        r->u = lr.u;
        r->v = lr.v;
        *inst = k;
        if (r->anyhit) return;
      }
    }
    return;
  }
  int front;
  if (r->anyhit)
    front = T->left_cheaper[node] ? 0 : 1;
  else
    front = r->d[T->axis[node]] > 0 ? 0 : 1;
  visit_top(W, first + front, r, inst);
  visit_top(W, first + 1 - front, r, inst);
}

static void world_trace(const orq_world* W, Ray* r, int* inst) {
  *inst = -1;
  if (!W->inner) {
    const Tree T = as_tree(W->top);
    visit(&T, 0, r);
  } else {
    visit_top(W, 0, r, inst);
  }
}

/* orq_trace over a world; inst = hit instance (-1: none / flat world). */
int orq_trace_world(const orq_world* W, int n, const float* org, const float* dir,
                    const float* tmax, int anyhit, int* hit, float* t, int* prim,
                    float* u, float* v, int* inst) {
  for (int i = 0; i < n; ++i) {
    Ray r;
    ray_init(&r, org, dir, n, i, tmax[i], anyhit);
    int k;
    world_trace(W, &r, &k);
    hit[i] = r.hit;
    t[i] = r.minT;
    prim[i] = r.hit ? r.prim : -1;
    u[i] = r.u;
    v[i] = r.v;
    if (inst) inst[i] = r.hit ? k : -1;
  }
  return 0;
}

/* Image coordinates of frame samples [i0, i1) (item = pixel * spp + s):
 * spp == 1 the SingleSampler pixel centres, otherwise stratified jitter
 * (strata x strata cells, PCG32 keyed by seed and item) - the sampling of
 * rfmanta_b200/csrc/rq_instance.cu sample_ray. */
static void sample_coords(int xres, int yres, int spp, uint64_t seed, long long item,
                          float* px, float* py) {
  const long long pix = item / spp;
  const int s = (int)(item - pix * spp);
  const int x = (int)(pix % xres), y = (int)(pix / xres);
  const float xscale = (float)2 / xres;
  const float yscale = (float)2 / yres;
  if (spp == 1) {
    const float xoffset = (-xres / (float)2 + (float)0.5) * xscale;
    const float yoffset = (-yres / (float)2 + (float)0.5) * yscale;
    *px = (float)x * xscale + xoffset;
    *py = (float)y * yscale + yoffset;
    return;
  }
  int strata = 1;
  while (strata * strata < spp) ++strata;
  Pcg32 g;
  pcg_seed(&g, seed ^ ((uint64_t)item * 0x9E3779B97F4A7C15ULL), (uint64_t)item);
  const float jx = ((float)(s % strata) + pcg_float(&g)) / (float)strata;
  const float jy = ((float)(s / strata) + pcg_float(&g)) / (float)strata;
  *px = ((float)x + jx) * xscale + ((float)(-xres) / 2.f) * xscale;
  *py = ((float)y + jy) * yscale + ((float)(-yres) / 2.f) * yscale;
}

void orq_sample_coords(int xres, int yres, int spp, unsigned long long seed, long long i0,
                       long long i1, float* px, float* py) {
  for (long long i = i0; i < i1; ++i)
    sample_coords(xres, yres, spp, seed, i, &px[i - i0], &py[i - i0]);
}

/* One Whitted sample (the body of orq_render_whitted) at image coordinates
 * (px, py) over a world; returns the shadow rays sent. */
/* ipow (Core/Math/ipow.h:21-31). */
static float ipow_f(float x, int p) {
  float result = 1;
  while (p) {
    if (p & 1) result *= x;
    x *= x;
    p >>= 1;
  }
  return result;
}

/* Material m is a Phong (Model/Materials/Phong.cc:130-410, scalar branch,
 * no reflection) when mat_pow is given and mat_pow[m] >= 0, else a
 * Lambertian. */
/* How a frame shades: material tables, lights, and the recursion limits of
 * reflective Phong (RenderParameters::maxDepth / importanceCutoff,
 * Interface/RenderParameters.h:11-15). */
typedef struct {
  const float* mat_rgb;
  const float* mat_spec;
  const int* mat_pow;    /* >= 0: Phong with that exponent */
  const float* mat_refl; /* Phong reflectivity (NULL = none) */
  const float* lights;
  int nl;
  const float* ambient;
  const float* background;
  int max_depth;
  float cutoff;
  const orq_env* env;
} Shading;

/* Raytracer::traceRays for one ray (Engine/Renderers/Raytracer.cc:49-97):
 * the closest hit shaded by its material - Lambertian::shade, or
 * Phong::shade (Model/Materials/Phong.cc:130-540, scalar branches) whose
 * reflection, when its reflectivity is not 0 and depth < maxDepth, traces
 * the mirrored ray d - N (2 N.d) from the hit point with importance x
 * reflectivity if that importance's luminance exceeds the cutoff (else its
 * colour is black) and adds its colour x reflectivity - with HardShadows
 * shadow rays to every point light; the background where nothing is hit.
 * Returns the shadow rays sent; *kout is the hit instance. */
static long long trace_color(const orq_world* W, const Shading* S, Ray* r, int depth,
                             const float* imp, float* rgb, int* kout) {
  int k;
  world_trace(W, r, &k);
  *kout = k;
  if (!r->hit) {
    env_background(S->env, S->background, r->d, rgb);
    return 0;
  }
  const orq_tree* HT = W->inner ? &W->inner[W->inst_scene[k]] : W->top;
  const Tree T = as_tree(HT);
  const unsigned m = HT->face_mat[r->prim];
  const float* kd = S->mat_rgb + 3 * m;
  const int phong = S->mat_pow && S->mat_pow[m] >= 0;
  float spec[3] = {0.f, 0.f, 0.f};
  float nrm[3];
  tri_normal(&T, r->prim, nrm);
  float ffn[3];
  const float dn = nrm[0] * r->d[0] + nrm[1] * r->d[1] + nrm[2] * r->d[2];
  for (int c = 0; c < 3; ++c) ffn[c] = (dn <= 0) ? nrm[c] : -nrm[c];
  float total[3];
  env_ambient(S->env, S->ambient, r->d, ffn, total);
  float hp[3];
  for (int c = 0; c < 3; ++c) hp[c] = r->o[c] + r->d[c] * r->minT;
  long long shadow_rays = 0;
  for (int j = 0; j < S->nl; ++j) {
    const float* L = S->lights + 6 * j;
    float sd[3] = {L[0] - hp[0], L[1] - hp[1], L[2] - hp[2]};
    if (!(sd[0] * ffn[0] + sd[1] * ffn[1] + sd[2] * ffn[2] > 0)) continue;
    Ray s;
    for (int c = 0; c < 3; ++c) {
      s.o[c] = hp[c];
      s.d[c] = sd[c];
      s.inv[c] = (float)1 / sd[c];
    }
    s.minT = 1 - T_EPSILON;
    s.hit = 0;
    s.prim = -1;
    s.u = s.v = 0.f;
    s.anyhit = 1;
    s.node_tests = s.tri_tests = 0;
    shadow_rays++;
    int sk;
    world_trace(W, &s, &sk);
    if (s.hit) continue;
    float sum = 0;
    for (int c = 0; c < 3; ++c) sum += sd[c] * sd[c];
    float scale = 1 / sqrtf(sum);
    for (int c = 0; c < 3; ++c) sd[c] *= scale;
    const float cos_theta = sd[0] * ffn[0] + sd[1] * ffn[1] + sd[2] * ffn[2];
    for (int c = 0; c < 3; ++c) total[c] += L[3 + c] * cos_theta;
    if (phong) {
      const float H[3] = {sd[0] - r->d[0], sd[1] - r->d[1], sd[2] - r->d[2]};
      const float cos_alpha = H[0] * ffn[0] + H[1] * ffn[1] + H[2] * ffn[2];
      if (cos_alpha > 0) {
        const float length = sqrtf(H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
        const float scale = ipow_f(cos_alpha / length, S->mat_pow[m]);
        for (int c = 0; c < 3; ++c) spec[c] += L[3 + c] * scale;
      }
    }
  }
  if (phong) {
    const float* ks = S->mat_spec + 3 * m;
    for (int c = 0; c < 3; ++c) rgb[c] = spec[c] * ks[c] + total[c] * kd[c];
  } else {
    for (int c = 0; c < 3; ++c) rgb[c] = total[c] * kd[c];
  }
  const float refl = (phong && S->mat_refl) ? S->mat_refl[m] : 0.f;
  if (refl != 0.f && depth < S->max_depth) {
    float cimp[3], child[3] = {0.f, 0.f, 0.f};
    for (int c = 0; c < 3; ++c) cimp[c] = imp[c] * refl;
    const float lum = cimp[0] * 0.3f + cimp[1] * 0.59f + cimp[2] * 0.11f;
    if (lum > S->cutoff) {
      Ray q;
      const float s2 = 2 * (ffn[0] * r->d[0] + ffn[1] * r->d[1] + ffn[2] * r->d[2]);
      for (int c = 0; c < 3; ++c) {
        q.o[c] = hp[c];
        q.d[c] = r->d[c] - ffn[c] * s2;
        q.inv[c] = (float)1 / q.d[c];
      }
      q.minT = MAXT;
      q.hit = 0;
      q.prim = -1;
      q.u = q.v = 0.f;
      q.anyhit = 0;
      q.node_tests = q.tri_tests = 0;
      int qk;
      shadow_rays += trace_color(W, S, &q, depth + 1, cimp, child, &qk);
    }
    for (int c = 0; c < 3; ++c) rgb[c] = rgb[c] + child[c] * refl;
  }
  return shadow_rays;
}

/* One image sample: the camera ray through (px, py) traced and shaded. */
static long long whitted_sample(const orq_world* W, const Shading* S, const float* cam,
                                float px, float py, float* rgb, float* tprim, int* prim) {
  Ray r;
  const float* dir = cam + 3;
  const float* cu = cam + 6;
  const float* cv = cam + 9;
  for (int c = 0; c < 3; ++c) {
    r.o[c] = cam[c];
    r.d[c] = cv[c] * px + cu[c] * py + dir[c];
  }
  v_normalize(r.d);
  for (int c = 0; c < 3; ++c) r.inv[c] = (float)1 / r.d[c];
  r.minT = MAXT;
  r.hit = 0;
  r.prim = -1;
  r.u = r.v = 0.f;
  r.anyhit = 0;
  r.node_tests = r.tri_tests = 0;
  const float one[3] = {1.f, 1.f, 1.f};
  int k;
  const long long n = trace_color(W, S, &r, 0, one, rgb, &k);
  *tprim = r.minT;
  *prim = r.hit ? r.prim : -1;
  return n;
}

/* Supersampled Whitted frame over a world (Lambertian and Phong materials,
 * reflective ones up to max_depth, see trace_color), pixel rows [y0, y1): per pixel
 * the spp samples' colours summed in sample order and scaled by 1/spp.
 * Optional per-sample outputs (indexed by item - y0 * xres * spp): colour,
 * primary t and triangle id.  Returns the shadow rays sent. */
long long orq_render_frame(const orq_world* W, const float* mat_rgb, const float* mat_spec,
                           const int* mat_pow, const float* mat_refl, int max_depth,
                           float cutoff, const float* cam,
                           int xres, int yres, int spp, unsigned long long seed,
                           const float* lights, int nl, const float* ambient,
                           const float* background, int y0, int y1, float* rgb,
                           float* sample_rgb, float* sample_t, int* sample_prim,
                           const orq_env* env) {
  const Shading S = {mat_rgb, mat_spec, mat_pow, mat_refl, lights, nl, ambient, background,
                     max_depth, cutoff, env};
  long long shadow = 0;
  const float inv = (float)1 / (float)spp;
  for (int y = y0; y < y1; ++y)
    for (int x = 0; x < xres; ++x) {
      const long long pix = (long long)y * xres + x;
      float acc[3] = {0.f, 0.f, 0.f};
      for (int s = 0; s < spp; ++s) {
        const long long item = pix * spp + s;
        const long long o = item - (long long)y0 * xres * spp;
        float px, py, c[3], t;
        int p;
        sample_coords(xres, yres, spp, seed, item, &px, &py);
        shadow += whitted_sample(W, &S, cam, px, py, c, &t, &p);
        for (int j = 0; j < 3; ++j) acc[j] += c[j];
        if (sample_rgb)
          for (int j = 0; j < 3; ++j) sample_rgb[3 * o + j] = c[j];
        if (sample_t) sample_t[o] = t;
        if (sample_prim) sample_prim[o] = p;
      }
      const long long po = pix - (long long)y0 * xres;
      for (int j = 0; j < 3; ++j) rgb[3 * po + j] = acc[j] * inv;
    }
  return shadow;
}
