// Two-level (instanced) scenes: creation, ray queries, and the
// supersampled Whitted frame that runs over flat or instanced scenes.
//
// A Manta scene whose top-level DynBVH sits over InstanceT objects
// (Model/Instances/InstanceT.cc) - translated copies of inner DynBVH
// objects - maps to an instanced rq_scene: the inner scenes are ordinary
// rq_scenes, the top-level tree is built by the GPU builder over the
// instances' boxes (InstanceT::computeBounds: inner bounds + translation).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_instance.cuh"
#include "rq_pathcore.cuh"
#include "rq_render.h"
#include "rq_scene.h"

namespace rq {

int gpu_build(Scene* s, HostTree& out, double* seconds);

static int ifail(int code, const std::string& m) {
  set_error(m);
  return code;
}

static float bits_as_float(int32_t i) {
  float f;
  std::memcpy(&f, &i, 4);
  return f;
}

// ------------------------------------------------------------ queries ----

template <int KIND, bool ANY>
__global__ void __launch_bounds__(128)
    trace2_kernel(DevScene T, const DevScene* blas, RayArgs a, int32_t* inst) {
  extern __shared__ int2 smem_stack[];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  Ray r;
  const int n = a.stride ? a.stride : a.n;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r.o[c] = __ldg(a.org + (size_t)c * n + i);
    r.d[c] = __ldg(a.dir + (size_t)c * n + i);
    r.inv[c] = fdiv(1.f, r.d[c]);
  }
  r.minT = __ldg(a.tmax + i);
  Hit h;
  int ih, bh;
  trace_two_level<KIND, ANY>(T, blas, r, h, ih, bh, smem_stack + threadIdx.x, blockDim.x);
  if (a.t) a.t[i] = h.t;
  if (a.prim) a.prim[i] = h.id;
  if (a.u) a.u[i] = h.u;
  if (a.v) a.v[i] = h.v;
  if (inst) inst[i] = ih;
}

cudaError_t launch_trace2(const Scene& s, const RayArgs& a, bool anyhit, int32_t* inst,
                          cudaStream_t st) {
  if (a.n <= 0) return cudaSuccess;
  const DevScene T = s.dev();
  const int bs = 128;
  const size_t smem = (size_t)(T.depth + s.max_blas_depth + 1) * bs * sizeof(int2);
  const int grid = (a.n + bs - 1) / bs;
  const void* f = s.tri_kind == kWald
                      ? (anyhit ? (const void*)trace2_kernel<kWald, true>
                                : (const void*)trace2_kernel<kWald, false>)
                      : (anyhit ? (const void*)trace2_kernel<kKS, true>
                                : (const void*)trace2_kernel<kKS, false>);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (s.tri_kind == kWald) {
    if (anyhit) trace2_kernel<kWald, true><<<grid, bs, smem, st>>>(T, s.d_blas, a, inst);
    else trace2_kernel<kWald, false><<<grid, bs, smem, st>>>(T, s.d_blas, a, inst);
  } else {
    if (anyhit) trace2_kernel<kKS, true><<<grid, bs, smem, st>>>(T, s.d_blas, a, inst);
    else trace2_kernel<kKS, false><<<grid, bs, smem, st>>>(T, s.d_blas, a, inst);
  }
  return cudaGetLastError();
}

// Lays out the top-level tree of an instanced scene: node records as for a
// triangle scene, and per leaf slot an instance record instead of a triangle
// record.
int set_instance_tree(Scene* s, const HostTree& t) {
  const int n_inst = (int)s->inst_blas.size();
  TreeLayout L;
  int rc = layout_tree(t, n_inst, L);
  if (rc != RQ_OK) return rc;
  std::vector<float4> recs(2 * std::max<size_t>(L.perm.size(), 1));
  for (size_t j = 0; j < L.perm.size(); ++j) {
    const int tag = L.perm[j];
    const int k = tag & 0x7fffffff;
    const float* T = s->inst_translation.data() + 3 * (size_t)k;
    recs[2 * j] = make_float4(T[0], T[1], T[2], bits_as_float(s->inst_blas[k]));
    recs[2 * j + 1] = make_float4(bits_as_float(tag), bits_as_float(s->inst_kind[k]), 0.f, 0.f);
  }
  s->free_tree();
  const size_t nrec = std::max<size_t>(L.recs.size(), 4);
  if (cudaMalloc(&s->d_nodes, nrec * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&s->d_tris, recs.size() * sizeof(float4)) != cudaSuccess)
    return ifail(RQ_ERR_OOM, "top-level tree");
  if (!L.recs.empty() &&
      cudaMemcpy(s->d_nodes, L.recs.data(), L.recs.size() * sizeof(float4),
                 cudaMemcpyHostToDevice) != cudaSuccess)
    return ifail(RQ_ERR_CUDA, "top-level tree upload");
  if (cudaMemcpy(s->d_tris, recs.data(), recs.size() * sizeof(float4), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return ifail(RQ_ERR_CUDA, "instance records upload");
  s->tree = t;
  s->n_records = L.n_records;
  s->n_leaves = L.n_leaves;
  s->n_leaf_tris = (int)L.perm.size();
  s->root_ref = L.root_ref;
  for (int c = 0; c < 3; ++c) {
    s->root_lo[c] = L.root_lo[c];
    s->root_hi[c] = L.root_hi[c];
  }
  s->depth = L.depth;
  s->has_tree = true;
  ++s->generation;
  return RQ_OK;
}

}  // namespace rq

extern "C" {

int rq_scene_create_instanced(rq_scene* const* inner, int n_inner, const int32_t* inst_scene,
                              const float* inst_translation, const int32_t* inst_kind,
                              int n_instances, rq_scene** out) {
  using namespace rq;
  if (!out) return ifail(RQ_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!inner || n_inner <= 0 || n_inner > 1024) return ifail(RQ_ERR_ARG, "1..1024 inner scenes");
  if (!inst_scene || !inst_translation || n_instances <= 0)
    return ifail(RQ_ERR_ARG, "no instances");
  const Scene* b0 = inner[0];
  if (!b0) return ifail(RQ_ERR_ARG, "NULL inner scene");
  std::vector<DevScene> ds(n_inner);
  int maxd = 0;
  for (int i = 0; i < n_inner; ++i) {
    const Scene* b = inner[i];
    if (!b || !b->has_tree) return ifail(RQ_ERR_STATE, "inner scene without a tree");
    if (b->instanced) return ifail(RQ_ERR_ARG, "inner scenes must be triangle meshes");
    if (b->device != b0->device || b->tri_kind != b0->tri_kind)
      return ifail(RQ_ERR_ARG, "inner scenes must share device and triangle kind");
    ds[i] = b->dev();
    maxd = std::max(maxd, ds[i].depth);
  }
  for (int k = 0; k < n_instances; ++k) {
    if (inst_scene[k] < 0 || inst_scene[k] >= n_inner)
      return ifail(RQ_ERR_ARG, "instance refers to a missing inner scene");
    const int kind = inst_kind ? inst_kind[k] : RQ_INST_TRANSLATE;
    if (kind != RQ_INST_TRANSLATE && kind != RQ_INST_NESTED)
      return ifail(RQ_ERR_ARG, "unknown instance kind");
    if (kind == RQ_INST_NESTED)
      for (int c = 0; c < 3; ++c)
        if (inst_translation[3 * k + c] != 0.f)
          return ifail(RQ_ERR_ARG, "a nested instance has no translation");
  }
  if (cudaSetDevice(b0->device) != cudaSuccess) return ifail(RQ_ERR_CUDA, "cudaSetDevice");
  // Instance boxes, InstanceT::computeBounds (InstanceT.cc:51-57): the
  // inner object's bounds (Mesh::computeBounds over all its vertices,
  // Model/Groups/Mesh.cc:195-225) moved by the translation; as degenerate
  // triangles (lo, hi, lo) whose bounding boxes are those boxes.
  std::vector<float> verts(9 * (size_t)n_instances);
  std::vector<uint32_t> idx(3 * (size_t)n_instances);
  std::vector<float> vb(6 * (size_t)n_inner);
  for (int i = 0; i < n_inner; ++i) {
    const std::vector<float>* hv = inner[i]->host_vertices();
    if (!hv) return ifail(RQ_ERR_CUDA, "reading an inner scene's vertices");
    const std::vector<float>& v = *hv;
    for (int c = 0; c < 3; ++c) {
      vb[6 * i + c] = v[c];
      vb[6 * i + 3 + c] = v[c];
    }
    for (size_t j = 3; j < v.size(); j += 3)
      for (int c = 0; c < 3; ++c) {
        const float x = v[j + c];
        if (x < vb[6 * i + c]) vb[6 * i + c] = x;
        if (x > vb[6 * i + 3 + c]) vb[6 * i + 3 + c] = x;
      }
  }
  for (int k = 0; k < n_instances; ++k) {
    const float* b = vb.data() + 6 * inst_scene[k];
    for (int c = 0; c < 3; ++c) {
      const float lo = b[c] + inst_translation[3 * k + c];
      const float hi = b[3 + c] + inst_translation[3 * k + c];
      verts[9 * k + c] = lo;
      verts[9 * k + 3 + c] = hi;
      verts[9 * k + 6 + c] = lo;
    }
    for (int j = 0; j < 3; ++j) idx[3 * k + j] = 3 * k + j;
  }
  std::unique_ptr<rq_scene> s(new rq_scene());
  s->device = b0->device;
  s->tri_kind = b0->tri_kind;
  s->num_sms = b0->num_sms;
  s->n_tris = n_instances;
  s->n_verts = 3 * n_instances;
  s->verts = verts;
  s->idx = idx;
  s->instanced = true;
  for (int i = 0; i < n_inner; ++i) {
    s->blas.push_back(inner[i]);
    s->blas_generation.push_back(inner[i]->generation);
  }
  s->inst_blas.assign(inst_scene, inst_scene + n_instances);
  s->inst_translation.assign(inst_translation, inst_translation + 3 * (size_t)n_instances);
  s->inst_kind.assign(n_instances, RQ_INST_TRANSLATE);
  if (inst_kind) s->inst_kind.assign(inst_kind, inst_kind + n_instances);
  s->max_blas_depth = maxd;
  for (int k = 0; k < 4; ++k) {
    s->cfg[k].block_threads = 128;
    s->cfg[k].blocks_per_sm = 0;
    s->cfg[k].refill_threshold = 8;
    s->cfg[k].persistent = 0;
    s->cfg[k].reg_stack = 0;
    s->cfg[k].node_layout = RQ_LAYOUT_DFS;
  }
  if (cudaMalloc(&s->d_verts, verts.size() * 4) != cudaSuccess ||
      cudaMalloc(&s->d_idx, idx.size() * 4) != cudaSuccess ||
      cudaMalloc(&s->d_blas, sizeof(DevScene) * n_inner) != cudaSuccess)
    return ifail(RQ_ERR_OOM, "instance boxes");
  if (cudaMemcpy(s->d_verts, verts.data(), verts.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->d_idx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->d_blas, ds.data(), sizeof(DevScene) * n_inner, cudaMemcpyHostToDevice) !=
          cudaSuccess)
    return ifail(RQ_ERR_CUDA, "instance upload");
  HostTree t;
  int rc = gpu_build(s.get(), t, &s->last_build_seconds);
  if (rc != RQ_OK) return rc;
  rc = s->set_tree(t);
  if (rc != RQ_OK) return rc;
  *out = s.release();
  return RQ_OK;
}

int rq_trace_device_ex(rq_scene* scene, int n, const float* d_org, const float* d_dir,
                       const float* d_tmax, int flags, float* d_t, int32_t* d_prim, float* d_u,
                       float* d_v, int32_t* d_inst, void* stream) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s) return rq::ifail(RQ_ERR_ARG, "NULL scene");
  if (!s->instanced) {
    if (d_inst && n > 0 && cudaMemsetAsync(d_inst, 0xff, 4 * (size_t)n,
                                           static_cast<cudaStream_t>(stream)) != cudaSuccess)
      return rq::ifail(RQ_ERR_CUDA, "instance output");
    return rq_trace_device(scene, n, d_org, d_dir, d_tmax, flags, d_t, d_prim, d_u, d_v, stream);
  }
  if (n < 0 || (n > 0 && (!d_org || !d_dir || !d_tmax))) return rq::ifail(RQ_ERR_ARG, "bad ray arrays");
  if (flags != RQ_CLOSEST && flags != RQ_ANYHIT) return rq::ifail(RQ_ERR_ARG, "bad flags");
  if (cudaSetDevice(s->device) != cudaSuccess) return rq::ifail(RQ_ERR_CUDA, "cudaSetDevice");
  rq::RayArgs a{n, d_org, d_dir, d_tmax, d_t, d_prim, d_u, d_v};
  const cudaError_t e = rq::launch_trace2(*s, a, flags == RQ_ANYHIT, d_inst,
                                          static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return rq::ifail(RQ_ERR_CUDA, std::string("trace: ") + cudaGetErrorString(e));
  return RQ_OK;
}

}  // extern "C"

// ------------------------------------------------ supersampled frame ----
//
// Raytracer::traceEyeRays per sample (PinholeCamera -normalizeRays,
// Lambertian or non-reflective Phong, HardShadows, PointLight; the Whitted
// wavefront of rq_render.cu) with `spp` stratified jittered samples per
// pixel averaged in sample order, over a flat or an instanced scene.  With spp = 1 the
// samples sit at the pixel centres of the SingleSampler mapping and the
// frame equals rq_render_whitted bit for bit.

namespace rq {

struct SampleParams {
  int spp, strata;
  unsigned long long seed;
};

struct SampleBufs {
  float* t;
  int32_t* prim;
  int32_t* pos;
  int32_t* blas;
  float* col;  // 3 per sample
  int32_t* queue;
  int32_t* counters;
  unsigned long long* shadow;
  uint8_t* hit;     // per sample: the primary ray hit something
  int32_t* tiles;   // compaction scratch
};

__device__ __forceinline__ void sample_ray(const FrameParams& P, const SampleParams& Q,
                                           long long item, Ray& r) {
  const long long pix = item / Q.spp;
  const int s = (int)(item - pix * Q.spp);
  const int x = (int)(pix % P.xres), y = (int)(pix / P.xres);
  if (Q.spp == 1) {
    primary_ray(P, x, y, r);
    return;
  }
  Pcg32 rng;
  pcg32_seed(rng, Q.seed ^ ((unsigned long long)item * 0x9E3779B97F4A7C15ULL),
             (unsigned long long)item);
  const float jx = fdiv(fadd((float)(s % Q.strata), pcg32_float(rng)), (float)Q.strata);
  const float jy = fdiv(fadd((float)(s / Q.strata), pcg32_float(rng)), (float)Q.strata);
  const float xscale = fdiv(2.f, (float)P.xres);
  const float yscale = fdiv(2.f, (float)P.yres);
  const float px = fadd(fmul(fadd((float)x, jx), xscale), fmul(fdiv((float)(-P.xres), 2.f), xscale));
  const float py = fadd(fmul(fadd((float)y, jy), yscale), fmul(fdiv((float)(-P.yres), 2.f), yscale));
  float d[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r.o[c] = P.cam[c];
    d[c] = fadd(fadd(fmul(P.cam[9 + c], px), fmul(P.cam[6 + c], py)), P.cam[3 + c]);
  }
  const float l = __fsqrt_rn(fadd(fadd(fmul(d[0], d[0]), fmul(d[1], d[1])), fmul(d[2], d[2])));
  const float sc = fdiv(1.f, l);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r.d[c] = fmul(d[c], sc);
    r.inv[c] = fdiv(1.f, r.d[c]);
  }
  r.minT = kMaxT;
}

template <int KIND, bool TWO, bool ANY, bool STATS>
__device__ __forceinline__ void scene_trace(const DevScene& S, const DevScene* blas, Ray& r,
                                            Hit& h, int& bh, int2* stk, int stride,
                                            Counts* cnt) {
  if (TWO) {
    int ih;
    trace_two_level<KIND, ANY, STATS>(S, blas, r, h, ih, bh, stk, stride, cnt);
  } else {
    int ref, sp;
    if (STATS) cnt->boxes += 1;
    start_ray(S, r, h, ref, sp);
    while (ref != kDone) step<KIND, ANY, STATS>(S, r, h, ref, sp, stk, stride, cnt);
    bh = -1;
  }
}

// Adds a warp's test counts into dst[0..1] (one atomic per warp and counter).
__device__ __forceinline__ void add_counts(unsigned long long* dst, int a, int b) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31u) == 0) {
    atomicAdd(dst, (unsigned long long)a);
    atomicAdd(dst + 1, (unsigned long long)b);
  }
}

template <int KIND, bool TWO, bool STATS>
__global__ void __launch_bounds__(128)
    frame_primary_kernel(DevScene S, const DevScene* blas, FrameParams P, SampleParams Q,
                         SampleBufs B, int n_items, unsigned long long* stats) {
  extern __shared__ int2 smem_stack[];
  const unsigned lane = threadIdx.x & 31u;
  // each warp claims 32 consecutive samples at a time (one per lane), so
  // warps that finish early take more instead of a fixed share
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&B.counters[1], 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n_items) break;
    const int it = base + (int)lane;
    bool hit = false;
    Counts cnt;
    if (it < n_items) {
      Ray r;
      sample_ray(P, Q, it, r);
      Hit h;
      int bh;
      scene_trace<KIND, TWO, false, STATS>(S, blas, r, h, bh, smem_stack + threadIdx.x,
                                           blockDim.x, &cnt);
      B.t[it] = h.t;
      B.prim[it] = h.id;
      B.pos[it] = h.pos;
      B.blas[it] = bh;
      hit = h.id >= 0;
      if (!hit) {
        float bg[3];
        background_color(P.env, P.background, r.d, bg);
        for (int c = 0; c < 3; ++c) B.col[3 * (size_t)it + c] = bg[c];
      }
    }
    // the shade queue is compacted in sample order afterwards, so that the
    // shade stage's warps take neighbouring samples whatever order the
    // primary warps finished in
    if (it < n_items) B.hit[it] = hit ? 1 : 0;
    if (STATS) add_counts(stats, cnt.boxes, cnt.tris);
  }
}

// Shades one hit the way Lambertian::shade / Phong::shade do (ambient plus
// every unshadowed point light; Phong adds its specular highlight): the
// local colour in col, the face-forward normal and hit point for a
// reflection.  Returns the material's reflectivity (0 unless a reflective
// Phong).
template <int KIND, bool TWO, bool STATS>
__device__ __forceinline__ float shade_hit(const DevScene& S, const DevScene* blas,
                                           const FrameParams& P, const Ray& r, float t,
                                           int prim, int pos, int bh, int2* stk, int stride,
                                           Counts* cnt, int& nshadow, float* col, float* ffn,
                                           float* hp) {
  const float shadow_tmax = fsub(1.f, kTEpsilon);
  const DevScene& HS = TWO ? blas[bh] : S;
  const int mat = (int)__ldg(HS.face_material + prim);
  float ks[3] = {0.f, 0.f, 0.f};
  int specpow = -1;
  if (P.phong) {
    const float4 ph = __ldg(reinterpret_cast<const float4*>(P.phong) + mat);
    ks[0] = ph.x;
    ks[1] = ph.y;
    ks[2] = ph.z;
    specpow = __float_as_int(ph.w);
  }
  float spec[3] = {0.f, 0.f, 0.f};
  float nrm[3];
  record_normal<KIND>(HS, pos, nrm);
  const float dn = dot3(nrm, r.d);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ffn[c] = (dn <= 0.f) ? nrm[c] : -nrm[c];
    hp[c] = fadd(r.o[c], fmul(r.d[c], t));
  }
  float total[3];
  ambient_light(P.env, P.ambient, r.d, ffn, total);
  for (int j = 0; j < P.n_lights; ++j) {
    const float* L = P.lights + 6 * j;
    float sd[3] = {fsub(L[0], hp[0]), fsub(L[1], hp[1]), fsub(L[2], hp[2])};
    if (!(dot3(sd, ffn) > 0.f)) continue;
    Ray s;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      s.o[c] = hp[c];
      s.d[c] = sd[c];
      s.inv[c] = fdiv(1.f, sd[c]);
    }
    s.minT = shadow_tmax;
    ++nshadow;
    Hit sh;
    int sb;
    scene_trace<KIND, TWO, true, STATS>(S, blas, s, sh, sb, stk, stride, cnt);
    if (sh.id >= 0) continue;
    const float sum = fadd(fadd(fmul(sd[0], sd[0]), fmul(sd[1], sd[1])), fmul(sd[2], sd[2]));
    const float scale = fdiv(1.f, __fsqrt_rn(sum));
#pragma unroll
    for (int c = 0; c < 3; ++c) sd[c] = fmul(sd[c], scale);
    const float cos_theta = dot3(sd, ffn);
#pragma unroll
    for (int c = 0; c < 3; ++c) total[c] = fadd(total[c], fmul(L[3 + c], cos_theta));
    if (specpow >= 0) {
      // Phong::shade scalar branch (Phong.cc:367-383): H = L - d,
      // ipow(Dot(H, N) / |H|, exponent) (Core/Math/ipow.h:21-31)
      const float H[3] = {fsub(sd[0], r.d[0]), fsub(sd[1], r.d[1]), fsub(sd[2], r.d[2])};
      const float cos_alpha = dot3(H, ffn);
      if (cos_alpha > 0.f) {
        const float len = __fsqrt_rn(dot3(H, H));
        float x = fdiv(cos_alpha, len), sc = 1.f;
        for (int pw = specpow; pw; pw >>= 1) {
          if (pw & 1) sc = fmul(sc, x);
          x = fmul(x, x);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) spec[c] = fadd(spec[c], fmul(L[3 + c], sc));
      }
    }
  }
  const float* kd = P.materials + 3 * (size_t)mat;
  if (specpow >= 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) col[c] = fadd(fmul(spec[c], ks[c]), fmul(total[c], __ldg(kd + c)));
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) col[c] = fmul(total[c], __ldg(kd + c));
  }
  return (specpow >= 0 && P.refl) ? __ldg(P.refl + mat) : 0.f;
}

// Shades the queued primary hits.  REFL: reflective Phong materials are
// followed (Phong.cc:438-540): while the material reflects, depth <
// maxDepth and the reflected importance's luminance (0.3 r + 0.59 g +
// 0.11 b, Core/Color/RGBTraits.h:43-45) exceeds the cutoff, the mirrored
// ray d - N (2 N.d) is traced from the hit point and shaded in turn; the
// chain is then folded from its end, colour = local + child x reflectivity,
// in the reference's order (a reflection cut off by importance adds black
// x reflectivity).
template <int KIND, bool TWO, bool STATS, bool REFL>
__global__ void __launch_bounds__(128)
    frame_shade_kernel(DevScene S, const DevScene* blas, FrameParams P, SampleParams Q,
                       SampleBufs B, unsigned long long* stats) {
  extern __shared__ int2 smem_stack[];
  const int nq = *(volatile const int*)&B.counters[0];
  const unsigned lane = threadIdx.x & 31u;
  int2* stk = smem_stack + threadIdx.x;
  const int stride = blockDim.x;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&B.counters[2], 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= nq) break;
    const int qi = base + (int)lane;
    int nshadow = 0;
    Counts cnt;
    if (qi < nq) {
      const int it = B.queue[qi];
      Ray r;
      sample_ray(P, Q, it, r);
      float col[3], ffn[3], hp[3];
      const float refl = shade_hit<KIND, TWO, STATS>(S, blas, P, r, B.t[it], B.prim[it],
                                                     B.pos[it], B.blas[it], stk, stride, &cnt,
                                                     nshadow, col, ffn, hp);
      if (!REFL || refl == 0.f || P.max_depth <= 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) B.col[3 * (size_t)it + c] = col[c];
      } else {
        float loc[kMaxReflectDepth + 1][3];
        float rf[kMaxReflectDepth + 1];
        for (int c = 0; c < 3; ++c) loc[0][c] = col[c];
        rf[0] = refl;
        float imp[3] = {1.f, 1.f, 1.f};
        float d[3] = {r.d[0], r.d[1], r.d[2]};
        int depth = 0;
        bool black = false;
        for (;;) {
          if (rf[depth] == 0.f || depth >= P.max_depth) break;
          float ci[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) ci[c] = fmul(imp[c], rf[depth]);
          const float lum = fadd(fadd(fmul(ci[0], 0.3f), fmul(ci[1], 0.59f)), fmul(ci[2], 0.11f));
          if (!(lum > P.cutoff)) {
            black = true;
            break;
          }
          Ray q;
          const float s2 = fmul(2.f, dot3(ffn, d));
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            q.o[c] = hp[c];
            q.d[c] = fsub(d[c], fmul(ffn[c], s2));
            q.inv[c] = fdiv(1.f, q.d[c]);
          }
          q.minT = kMaxT;
          Hit qh;
          int qb;
          scene_trace<KIND, TWO, false, STATS>(S, blas, q, qh, qb, stk, stride, &cnt);
          ++depth;
#pragma unroll
          for (int c = 0; c < 3; ++c) imp[c] = ci[c];
          if (qh.id < 0) {
            background_color(P.env, P.background, q.d, loc[depth]);
            rf[depth] = 0.f;
            break;
          }
          rf[depth] = shade_hit<KIND, TWO, STATS>(S, blas, P, q, qh.t, qh.id, qh.pos, qb, stk,
                                                  stride, &cnt, nshadow, loc[depth], ffn, hp);
#pragma unroll
          for (int c = 0; c < 3; ++c) d[c] = q.d[c];
        }
        float c3[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          c3[c] = black ? fadd(loc[depth][c], fmul(0.f, rf[depth])) : loc[depth][c];
        for (int k = depth - 1; k >= 0; --k)
#pragma unroll
          for (int c = 0; c < 3; ++c) c3[c] = fadd(loc[k][c], fmul(c3[c], rf[k]));
#pragma unroll
        for (int c = 0; c < 3; ++c) B.col[3 * (size_t)it + c] = c3[c];
      }
    }
    int tot = nshadow;
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0 && tot) atomicAdd(B.shadow, (unsigned long long)tot);
    if (STATS) add_counts(stats + 2, cnt.boxes, cnt.tris);
  }
}

__global__ void frame_resolve_kernel(SampleParams Q, SampleBufs B, int npix, float* rgb) {
  const float inv = fdiv(1.f, (float)Q.spp);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < npix; k += gridDim.x * blockDim.x) {
    float acc[3] = {0.f, 0.f, 0.f};
    for (int s = 0; s < Q.spp; ++s)
      for (int c = 0; c < 3; ++c) acc[c] = fadd(acc[c], B.col[3 * ((size_t)k * Q.spp + s) + c]);
    for (int c = 0; c < 3; ++c) rgb[3 * (size_t)k + c] = fmul(acc[c], inv);
  }
}

template <int KIND, bool TWO, bool STATS>
static cudaError_t frame_go(const Scene& s, const FrameParams& P, const SampleParams& Q,
                            const SampleBufs& B, int npix, float* rgb, cudaStream_t st,
                            const cudaEvent_t* ev, int nev) {
  const DevScene S = s.dev();
  const int bs = 128;
  const size_t smem = (size_t)(S.depth + (TWO ? s.max_blas_depth : 0) + 1) * bs * sizeof(int2);
  const bool refl = P.refl != nullptr;
  const void* f1 = (const void*)frame_primary_kernel<KIND, TWO, STATS>;
  const void* f2 = refl ? (const void*)frame_shade_kernel<KIND, TWO, STATS, true>
                        : (const void*)frame_shade_kernel<KIND, TWO, STATS, false>;
  if (smem > 48 * 1024) {
    cudaFuncSetAttribute(f1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(f2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  int a = 1, b = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, f1, bs, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f2, bs, smem);
  const int grid = std::max(1, std::min(a, b) * s.num_sms);
  const int n_items = npix * Q.spp;
  cudaError_t e = cudaMemsetAsync(B.counters, 0, 4 * sizeof(int), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(B.shadow, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  if (nev > 0) cudaEventRecord(ev[0], st);
  frame_primary_kernel<KIND, TWO, STATS>
      <<<std::max(1, std::min(grid, (n_items + bs - 1) / bs)), bs, smem, st>>>(
          S, s.d_blas, P, Q, B, n_items, s.stats);
  e = launch_flag_compaction(B.hit, n_items, B.tiles, &B.counters[0], B.queue, st);
  if (e != cudaSuccess) return e;
  if (nev > 1) cudaEventRecord(ev[1], st);
  if (refl)
    frame_shade_kernel<KIND, TWO, STATS, true><<<grid, bs, smem, st>>>(S, s.d_blas, P, Q, B,
                                                                      s.stats);
  else
    frame_shade_kernel<KIND, TWO, STATS, false><<<grid, bs, smem, st>>>(S, s.d_blas, P, Q, B,
                                                                       s.stats);
  if (nev > 2) cudaEventRecord(ev[2], st);
  frame_resolve_kernel<<<std::max(1, std::min(grid, (npix + 255) / 256)), 256, 0, st>>>(Q, B, npix, rgb);
  if (nev > 3) cudaEventRecord(ev[3], st);
  return cudaGetLastError();
}

template <int KIND, bool TWO>
static cudaError_t frame_go_any(const Scene& s, const FrameParams& P, const SampleParams& Q,
                                const SampleBufs& B, int npix, float* rgb, cudaStream_t st) {
  return s.stats ? frame_go<KIND, TWO, true>(s, P, Q, B, npix, rgb, st, s.stage_events,
                                             s.n_stage_events)
                 : frame_go<KIND, TWO, false>(s, P, Q, B, npix, rgb, st, s.stage_events,
                                              s.n_stage_events);
}

// Scratch of the supersampled frame, owned by the scene.
struct SampleScratch {
  size_t items = 0;
  SampleBufs B{};
  float* materials = nullptr;
  std::vector<float> host_materials;
  float4* phong = nullptr;
  std::vector<float4> host_phong;
  float* refl = nullptr;
  std::vector<float> host_refl;
  float* d_rgb = nullptr;
  size_t rgb_pix = 0;
  cudaStream_t stream = nullptr;
  void free_items() {
    cudaFree(B.t); cudaFree(B.prim); cudaFree(B.pos); cudaFree(B.blas); cudaFree(B.col);
    cudaFree(B.queue);
    cudaFree(B.hit);
    cudaFree(B.tiles);
    B.t = B.col = nullptr;
    B.prim = B.pos = B.blas = B.queue = B.tiles = nullptr;
    B.hit = nullptr;
    items = 0;
  }
  ~SampleScratch() {
    free_items();
    cudaFree(B.counters);
    cudaFree(B.shadow);
    cudaFree(materials);
    cudaFree(phong);
    cudaFree(refl);
    cudaFree(d_rgb);
    if (stream) cudaStreamDestroy(stream);
  }
};

void destroy_sample_scratch(SampleScratch* p) { delete p; }

}  // namespace rq

namespace {

int frame_prepare(rq::Scene* s, const rq_frame_params* fp, rq::FrameParams& P,
                  rq::SampleParams& Q) {
  using namespace rq;
  if (!fp) return ifail(RQ_ERR_ARG, "NULL params");
  const rq_whitted_params* p = &fp->whitted;
  if (p->xres <= 0 || p->yres <= 0) return ifail(RQ_ERR_ARG, "bad resolution");
  const int strata = (int)std::lround(std::sqrt((double)fp->spp));
  if (fp->spp <= 0 || strata * strata != fp->spp || fp->spp > 1024)
    return ifail(RQ_ERR_ARG, "spp must be a perfect square <= 1024");
  if ((long long)p->xres * p->yres * fp->spp > (1LL << 30)) return ifail(RQ_ERR_ARG, "frame too large");
  if (p->n_lights < 0 || p->n_lights > kMaxLights || (p->n_lights > 0 && !p->lights))
    return ifail(RQ_ERR_ARG, "0..16 point lights");
  if (p->n_materials <= 0 || !p->material_rgb) return ifail(RQ_ERR_ARG, "no materials");
  const std::vector<Scene*> meshes = s->instanced ? s->blas : std::vector<Scene*>{s};
  for (const Scene* m : meshes)
    if (m->max_face_material >= p->n_materials)
      return ifail(RQ_ERR_ARG, "face_material past n_materials");
  if (!s->has_tree) return ifail(RQ_ERR_STATE, "scene has no tree");
  if (s->instanced) {
    const int rc = s->check_inner_current();
    if (rc != RQ_OK) return rc;
  }
  std::memset(&P, 0, sizeof(P));
  camera_basis(p->eye, p->lookat, p->up, p->hfov, p->vfov, P.cam);
  P.xres = p->xres;
  P.yres = p->yres;
  P.n_lights = p->n_lights;
  std::memcpy(P.lights, p->lights, sizeof(float) * 6 * p->n_lights);
  std::memcpy(P.ambient, p->ambient, sizeof(P.ambient));
  std::memcpy(P.background, p->background, sizeof(P.background));
  if (!environment_from(p->environment, P.env))
    return ifail(RQ_ERR_ARG, "bad environment (kind, or a zero background up)");
  Q.spp = fp->spp;
  Q.strata = strata;
  Q.seed = fp->seed;
  if (!s->samples) s->samples = new SampleScratch();
  SampleScratch* x = s->samples;
  const size_t items = (size_t)p->xres * p->yres * fp->spp;
  if (x->items < items) {
    x->free_items();
    SampleBufs& B = x->B;
    if (cudaMalloc(&B.t, 4 * items) != cudaSuccess || cudaMalloc(&B.prim, 4 * items) != cudaSuccess ||
        cudaMalloc(&B.pos, 4 * items) != cudaSuccess || cudaMalloc(&B.blas, 4 * items) != cudaSuccess ||
        cudaMalloc(&B.col, 12 * items) != cudaSuccess || cudaMalloc(&B.queue, 4 * items) != cudaSuccess ||
        cudaMalloc(&B.hit, items) != cudaSuccess ||
        cudaMalloc(&B.tiles, 4 * (size_t)flag_compaction_tiles((int)items)) != cudaSuccess) {
      x->free_items();
      return ifail(RQ_ERR_OOM, "frame sample buffers");
    }
    x->items = items;
  }
  if (!x->B.counters && (cudaMalloc(&x->B.counters, 16) != cudaSuccess ||
                         cudaMalloc(&x->B.shadow, 8) != cudaSuccess))
    return ifail(RQ_ERR_OOM, "frame counters");
  const float* mrgb = p->material_rgb;
  if ((int)x->host_materials.size() != 3 * p->n_materials ||
      std::memcmp(x->host_materials.data(), mrgb, sizeof(float) * 3 * p->n_materials) != 0) {
    cudaFree(x->materials);
    x->materials = nullptr;
    if (cudaMalloc(&x->materials, 12 * (size_t)p->n_materials) != cudaSuccess ||
        cudaMemcpy(x->materials, mrgb, 12 * (size_t)p->n_materials, cudaMemcpyHostToDevice) != cudaSuccess)
      return ifail(RQ_ERR_OOM, "materials");
    x->host_materials.assign(mrgb, mrgb + 3 * p->n_materials);
  }
  P.materials = x->materials;
  P.phong = nullptr;
  if (fp->material_specpow) {
    if (!fp->material_specular) return ifail(RQ_ERR_ARG, "material_specpow without material_specular");
    std::vector<float4> ph(p->n_materials);
    for (int m = 0; m < p->n_materials; ++m) {
      const int sp = fp->material_specpow[m];
      if (sp > 4096) return ifail(RQ_ERR_ARG, "Phong exponent above 4096");
      ph[m] = make_float4(fp->material_specular[3 * m], fp->material_specular[3 * m + 1],
                          fp->material_specular[3 * m + 2], bits_as_float(sp));
    }
    if (x->host_phong.size() != ph.size() ||
        std::memcmp(x->host_phong.data(), ph.data(), ph.size() * sizeof(float4)) != 0) {
      cudaFree(x->phong);
      x->phong = nullptr;
      if (cudaMalloc(&x->phong, ph.size() * sizeof(float4)) != cudaSuccess ||
          cudaMemcpy(x->phong, ph.data(), ph.size() * sizeof(float4), cudaMemcpyHostToDevice) !=
              cudaSuccess)
        return ifail(RQ_ERR_OOM, "Phong table");
      x->host_phong = ph;
    }
    P.phong = reinterpret_cast<const float*>(x->phong);
  }
  P.refl = nullptr;
  P.max_depth = 0;
  P.cutoff = 0.f;
  if (fp->material_reflectivity) {
    if (!fp->material_specpow) return ifail(RQ_ERR_ARG, "material_reflectivity needs Phong materials");
    if (fp->max_depth < 0 || fp->max_depth > kMaxReflectDepth)
      return ifail(RQ_ERR_ARG, "max_depth must be in [0, 32]");
    std::vector<float> rf(fp->material_reflectivity, fp->material_reflectivity + p->n_materials);
    if (x->host_refl != rf) {
      cudaFree(x->refl);
      x->refl = nullptr;
      if (cudaMalloc(&x->refl, rf.size() * sizeof(float)) != cudaSuccess ||
          cudaMemcpy(x->refl, rf.data(), rf.size() * sizeof(float), cudaMemcpyHostToDevice) !=
              cudaSuccess)
        return ifail(RQ_ERR_OOM, "reflectivity table");
      x->host_refl = rf;
    }
    P.refl = x->refl;
    P.max_depth = fp->max_depth;
    P.cutoff = fp->importance_cutoff;
  }
  return RQ_OK;
}

int frame_run(rq::Scene* s, const rq::FrameParams& P, const rq::SampleParams& Q, float* d_rgb,
              uint64_t* d_shadow, cudaStream_t st) {
  using namespace rq;
  SampleBufs B = s->samples->B;
  if (d_shadow) B.shadow = reinterpret_cast<unsigned long long*>(d_shadow);
  const int npix = P.xres * P.yres;
  cudaError_t e;
  if (s->tri_kind == kWald)
    e = s->instanced ? frame_go_any<kWald, true>(*s, P, Q, B, npix, d_rgb, st)
                     : frame_go_any<kWald, false>(*s, P, Q, B, npix, d_rgb, st);
  else
    e = s->instanced ? frame_go_any<kKS, true>(*s, P, Q, B, npix, d_rgb, st)
                     : frame_go_any<kKS, false>(*s, P, Q, B, npix, d_rgb, st);
  if (e != cudaSuccess) return ifail(RQ_ERR_CUDA, std::string("frame launch: ") + cudaGetErrorString(e));
  return RQ_OK;
}

}  // namespace

extern "C" {

int rq_render_frame_device(rq_scene* scene, const rq_frame_params* params, float* d_rgb,
                           uint64_t* d_shadow_rays, void* stream) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s || !d_rgb) return rq::ifail(RQ_ERR_ARG, "NULL argument");
  if (cudaSetDevice(s->device) != cudaSuccess) return rq::ifail(RQ_ERR_CUDA, "cudaSetDevice");
  std::lock_guard<std::mutex> g(s->frame_mu);
  rq::FrameParams P;
  rq::SampleParams Q;
  int rc = frame_prepare(s, params, P, Q);
  if (rc != RQ_OK) return rc;
  return frame_run(s, P, Q, d_rgb, d_shadow_rays, static_cast<cudaStream_t>(stream));
}

int rq_render_frame(rq_scene* scene, const rq_frame_params* params, float* rgb,
                    uint64_t* shadow_rays) {
  rq::Scene* s = reinterpret_cast<rq::Scene*>(scene);
  if (!s || !rgb) return rq::ifail(RQ_ERR_ARG, "NULL argument");
  if (cudaSetDevice(s->device) != cudaSuccess) return rq::ifail(RQ_ERR_CUDA, "cudaSetDevice");
  std::lock_guard<std::mutex> g(s->frame_mu);
  rq::FrameParams P;
  rq::SampleParams Q;
  int rc = frame_prepare(s, params, P, Q);
  if (rc != RQ_OK) return rc;
  rq::SampleScratch* x = s->samples;
  const size_t npix = (size_t)P.xres * P.yres;
  if (!x->stream && cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess)
    return rq::ifail(RQ_ERR_CUDA, "stream");
  if (x->rgb_pix < npix) {
    cudaFree(x->d_rgb);
    x->d_rgb = nullptr;
    if (cudaMalloc(&x->d_rgb, 12 * npix) != cudaSuccess) return rq::ifail(RQ_ERR_OOM, "image");
    x->rgb_pix = npix;
  }
  rc = frame_run(s, P, Q, x->d_rgb, nullptr, x->stream);
  if (rc != RQ_OK) return rc;
  unsigned long long ns = 0;
  cudaError_t e = cudaMemcpyAsync(rgb, x->d_rgb, 12 * npix, cudaMemcpyDeviceToHost, x->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&ns, x->B.shadow, 8, cudaMemcpyDeviceToHost, x->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(x->stream);
  if (e != cudaSuccess) return rq::ifail(RQ_ERR_CUDA, cudaGetErrorString(e));
  if (shadow_rays) *shadow_rays = ns;
  return RQ_OK;
}

}  // extern "C"
