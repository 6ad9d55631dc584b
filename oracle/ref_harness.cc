// Test infrastructure, not product code.
//
// Harness that drives the reference's own classes (compiled from the
// reference sources by oracle/ref.mk) through a small extern "C" surface so
// the Python tests and the CPU-baseline leg of bench.py can call them with
// plain arrays.  Nothing here restates an algorithm: every result comes out
// of the reference's code path.
//
//   scene      Mesh (Model/Groups/Mesh.h:27-102) of WaldTriangle
//              (Model/Primitives/WaldTriangle.cc:13-126) or
//              KenslerShirleyTriangle primitives, one Lambertian
//              (Model/Materials/Lambertian.cc) per material id, under a
//              DynBVH (Model/Groups/DynBVH.cc:1699 rebuild).
//   intersect  DynBVH::intersect (DynBVH.cc:101-272) over 64-ray packets
//              (Interface/RayPacket.h:58-130), closest hit or AnyHit.
//   render     Raytracer::traceEyeRays (Engine/Renderers/Raytracer.cc:41-97)
//              with PinholeCamera(-normalizeRays), Lambertian, HardShadows
//              (Engine/Shadows/HardShadows.cc:46), PointLight,
//              ConstantAmbient and ConstantBackground, on N pthreads that
//              take image rows from an atomic counter (the role of
//              Core/Thread/WorkQueue.cc:61-69 in the reference's frame loop).
//
// Compiled as C++98 (the reference's dialect).

#include <Core/Color/Color.h>
#include <Core/Exceptions/Exception.h>
#include <Core/Color/RGBColor.h>
#include <Core/Geometry/BBox.h>
#include <Core/Geometry/Vector.h>
#include <Core/Math/CheapRNG.h>
#include <Core/Thread/Barrier.h>
#include <Core/Thread/Thread.h>
#include <Engine/Renderers/KajiyaPathtracer.h>
#include <Engine/Renderers/Raytracer.h>
#include <Engine/SampleGenerators/UniformRandomGenerator.h>
#include <Model/Lights/AreaLight.h>
#include <Model/Primitives/Parallelogram.h>
#include <Engine/SampleGenerators/ConstantSampleGenerator.h>
#include <Engine/Shadows/HardShadows.h>
#include <Interface/Context.h>
#include <Interface/LightSet.h>
#include <Interface/RayPacket.h>
#include <Interface/Scene.h>
#include <Model/AmbientLights/ConstantAmbient.h>
#include <Model/AmbientLights/EyeAmbient.h>
#include <Model/Backgrounds/ConstantBackground.h>
#include <Model/Backgrounds/LinearBackground.h>
#include <Model/Cameras/PinholeCamera.h>
#include <Model/Groups/DynBVH.h>
#include <Model/Groups/Group.h>
#include <Model/Groups/Mesh.h>
#include <Model/Instances/InstanceT.h>
#include <Model/Instances/MPT.h>
#include <Model/Lights/PointLight.h>
#include <Model/Materials/Lambertian.h>
#include <Model/Materials/Phong.h>
#include <Model/Readers/PlyReader.h>
#include <Model/Groups/ObjGroup.h>
#include <Model/Materials/Dielectric.h>
#include <Model/Materials/Transparent.h>
#include <Model/Readers/glm/glm.h>
#include <Model/Textures/ImageTexture.h>
#include <Model/Primitives/KenslerShirleyTriangle.h>
#include <Model/Primitives/MeshTriangle.h>
#include <Model/Primitives/WaldTriangle.h>

#ifdef MREF_DROPIN
#include <rfmanta_b200/manta/GpuDynBVH.h>
#include <rfmanta_b200/manta/GpuHardShadows.h>
#include <rfmanta_b200/manta/GpuMeshPrimitive.h>
#endif

#include <pthread.h>
#include <unistd.h>
#include <stdio.h>
#include <string.h>
#include <sys/time.h>
#include <map>
#include <string>
#include <vector>

using namespace Manta;

namespace Manta {
// No image readers are built into the checker: an OBJ material's texture
// map fails to load and ObjGroup keeps its constant colour
// (Model/Groups/ObjGroup.cc:38-64).
ImageTexture<Color>* LoadColorImageTexture(const std::string& file_name, std::ostream*, bool) {
  throw InputError("image textures are not built into the checker: " + file_name);
}
}  // namespace Manta

namespace {

// Exposes the protected tree arrays and the SAH cost routine of the
// reference DynBVH (DynBVH.h:88-89, DynBVH.cc:3389-3416).
class ExposedBVH : public DynBVH {
public:
  ExposedBVH() : DynBVH(false), ray_counters(0) {}
  // When set, counts the unmasked rays of every intersect call per worker
  // (counters[16 * proc]) before handing the packet to DynBVH::intersect.
  long long* ray_counters;
  void intersect(const RenderContext& context, RayPacket& rays) const {
    if (ray_counters) {
      long long n = 0;
      for (int i = rays.begin(); i < rays.end(); ++i)
        if (!rays.rayIsMasked(i)) ++n;
      ray_counters[16 * context.proc] += n;
    }
    DynBVH::intersect(context, rays);
  }
  const std::vector<BVHNode>& treeNodes() const { return nodes; }
  const std::vector<int>& treeIds() const { return object_ids; }
  float sahCost() { return computeCost<true>(0); }
  // DynBVH::costs and DynBVH::nextFree (DynBVH.h:105, 382): the state the
  // tree rotations of the next update start from.
  const std::vector<Real>& treeCosts() const { return costs; }
  int nextFreeNode() const { return nextFree; }
};

// Reads MeshTriangle::myID (protected, Model/Primitives/MeshTriangle.h:63).
class TriId : public MeshTriangle {
public:
  static unsigned int of(const Primitive* p) {
    return static_cast<const TriId*>(static_cast<const MeshTriangle*>(p))->myID;
  }
};

// Exposes the camera basis set up by PinholeCamera::setup
// (Model/Cameras/PinholeCamera.cc:167-198).
class ExposedCamera : public PinholeCamera {
public:
  ExposedCamera(const std::vector<std::string>& args) : PinholeCamera(args) {}
  void basis(float* out) const {
    for (int i = 0; i < 3; ++i) {
      out[0 + i] = eye[i];
      out[3 + i] = direction[i];
      out[6 + i] = u[i];
      out[9 + i] = v[i];
    }
  }
};

// HardShadows that also counts the shadow rays it sends into the scene.
class CountingShadows : public HardShadows {
public:
  CountingShadows() : HardShadows(false) {}
  long long* counter;  // per-thread slot, set before each use
  void computeShadows(const RenderContext& context, StateBuffer& state,
                      const LightSet* lights, RayPacket& source,
                      RayPacket& shadow) {
    HardShadows::computeShadows(context, state, lights, source, shadow);
    for (int i = shadow.begin(); i < shadow.end(); ++i)
      if (!shadow.rayIsMasked(i)) ++*counter;
  }
};

#ifdef MREF_DROPIN
// GpuHardShadows that counts the shadow rays it hands out, as
// CountingShadows does for HardShadows.
class CountingGpuShadows : public GpuHardShadows {
public:
  explicit CountingGpuShadows(const GpuDynBVH* bvh) : GpuHardShadows(bvh), counter(0) {}
  long long* counter;
  void computeShadows(const RenderContext& context, StateBuffer& state,
                      const LightSet* lights, RayPacket& source,
                      RayPacket& shadow) {
    GpuHardShadows::computeShadows(context, state, lights, source, shadow);
    for (int i = shadow.begin(); i < shadow.end(); ++i)
      if (!shadow.rayIsMasked(i)) ++*counter;
  }
};
#endif

// Hands a packet to an InstanceT with the derived-data flags cleared.
// InstanceT::intersect (Model/Instances/InstanceT.cc:60-66) builds its local
// packet from rays.getAllFlags(); HaveInverseDirections / HaveSigns set by
// the enclosing DynBVH would then make the inner DynBVH::intersect skip
// computing inverse directions and signs for a packet whose data
// InstanceT never filled (it would read uninitialised memory).  Cleared,
// the inner DynBVH computes both itself (DynBVH.cc:116-120).  The flags are
// restored afterwards; the outer packet's data is untouched.
class InstanceGuard : public Object {
public:
  explicit InstanceGuard(InstanceT* it) : it(it) {}
  void computeBounds(const PreprocessContext& c, BBox& b) const { it->computeBounds(c, b); }
  void intersect(const RenderContext& c, RayPacket& rays) const {
    const int mask = RayPacket::HaveInverseDirections | RayPacket::HaveSigns |
                     RayPacket::ConstantSigns;
    const int saved = rays.getAllFlags() & mask;
    rays.resetFlag(mask);
    it->intersect(c, rays);
    rays.setFlag(saved);
  }
  InstanceT* it;
};

struct RefScene {
  Mesh* mesh;      // NULL for a two-level scene
  ExposedBVH* bvh;
  Object* object;  // what rays are traced against: bvh, or a drop-in
  std::vector<Material*> materials;
  std::vector<float> diffuse;  // rgb per mesh material
  LightSet* lights;
  Scene* scene;
  // two-level scenes: instance index of each top-level InstanceT object
  std::map<const Primitive*, int> instance_of;
  // renders' ambient light and background: kinds (0 constant, 1 EyeAmbient /
  // LinearBackground) and LinearBackground's cdown and up
  int env_ambient, env_background;
  float env_down[3], env_up[3];
  // drop-in builds: Whitted renders use GpuHardShadows (all lights' shadow
  // rays of a packet in one submission) instead of HardShadows
  int gpu_shadows;
};

// The ambient light and background a render of this scene uses: the given
// colours as ConstantAmbient / ConstantBackground, or EyeAmbient and
// LinearBackground(cup = colour, cdown, up) when the scene asks for them.
AmbientLight* make_ambient(const RefScene* s, const float* c) {
  if (s->env_ambient == 1) return new EyeAmbient(Color(RGB(c[0], c[1], c[2])));
  return new ConstantAmbient(Color(RGB(c[0], c[1], c[2])));
}

Background* make_background(const RefScene* s, const float* c) {
  if (s->env_background == 1)
    return new LinearBackground(Color(RGB(c[0], c[1], c[2])),
                                Color(RGB(s->env_down[0], s->env_down[1], s->env_down[2])),
                                Vector(s->env_up[0], s->env_up[1], s->env_up[2]));
  return new ConstantBackground(Color(RGB(c[0], c[1], c[2])));
}

// Triangle id (and instance index, -1 for none) of a hit: a hit on an
// InstanceT carries the inner primitive in its MPT scratchpad
// (Model/Instances/InstanceT.cc:80-87).
int hit_prim(const RefScene* s, RayPacket& rays, int i, int* inst) {
  const Primitive* p = rays.getHitPrimitive(i);
  if (!s->instance_of.empty()) {
    std::map<const Primitive*, int>::const_iterator it = s->instance_of.find(p);
    if (it != s->instance_of.end()) {
      if (inst) *inst = it->second;
      return (int)TriId::of(rays.scratchpad<MPT>(i).primitive);
    }
  }
  if (inst) *inst = -1;
  return (int)TriId::of(p);
}

double now_s() {
  struct timeval tv;
  gettimeofday(&tv, 0);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

}  // namespace

// The reference's thread library registers an atexit handler that calls
// ::exit(0) from inside process exit (Core/Thread/Thread_pthreads.cc:
// 596-655, 841-846, 874), which replaces the process's exit status with 0:
// a test run or benchmark that loaded this library would report success
// whatever failed.  (Thread::setCallExit(false) avoids the call but then
// process exit blocks in that handler.)  mref_keep_exit_status makes sure the
// thread library is initialised (a Barrier does that, Barrier_default.cc:
// 72-76), then registers an on_exit handler - run before every handler
// registered earlier - that flushes stdio and ends the process with the
// status exit() was given.
static void keep_exit_status(int status, void*) {
  fflush(NULL);
  _exit(status);
}

extern "C" {

void mref_keep_exit_status(void) {
  static bool done = false;
  if (done) return;
  done = true;
  if (!Thread::isInitialized()) {
    Barrier b("mref exit status");
  }
  on_exit(keep_exit_status, 0);
}

// Builds Mesh + triangles + DynBVH.  tri_kind 0 = WaldTriangle,
// 1 = KenslerShirleyTriangle.  mat_rgb holds nmat diffuse colours.
void* mref_scene_create(const float* verts, int nverts, const unsigned* idx,
                        int ntris, const unsigned* face_mat,
                        const float* mat_rgb, int nmat, int tri_kind) {
  try {
    RefScene* s = new RefScene();
    s->mesh = new Mesh();
    Mesh* m = s->mesh;
    m->vertices.resize(nverts);
    for (int i = 0; i < nverts; ++i)
      m->vertices[i] = Vector(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    m->vertex_indices.assign(idx, idx + 3 * (size_t)ntris);
    m->face_material.assign(face_mat, face_mat + ntris);
    s->diffuse.assign(mat_rgb, mat_rgb + 3 * nmat);
    for (int k = 0; k < nmat; ++k) {
      Material* mat = new Lambertian(
          Color(RGB(mat_rgb[3 * k], mat_rgb[3 * k + 1], mat_rgb[3 * k + 2])));
      m->materials.push_back(mat);
      s->materials.push_back(mat);
    }
    for (int t = 0; t < ntris; ++t) {
      if (tri_kind == 0)
        m->addTriangle(new WaldTriangle(m, t));
      else
        m->addTriangle(new KenslerShirleyTriangle(m, t));
    }
    s->lights = new LightSet();
    s->lights->setAmbientLight(new ConstantAmbient(Color(RGB(0, 0, 0))));
    s->scene = 0;
    PreprocessContext ctx;
    ctx.globalLights = s->lights;
    m->preprocess(ctx);
    s->bvh = new ExposedBVH();
    s->bvh->setGroup(m);
    s->bvh->rebuild(0, 1);
    s->object = s->bvh;
    return s;
  } catch (...) {
    return 0;
  }
}

// RenderParameters::maxDepth and importanceCutoff of the scene's renders
// (Interface/RenderParameters.h: 15 and 0.01 unless set).
// Ambient light and background kinds for this scene's later renders.
int mref_scene_set_environment(void* h, int ambient_kind, int background_kind,
                               const float* down, const float* up) {
  RefScene* s = static_cast<RefScene*>(h);
  s->env_ambient = ambient_kind;
  s->env_background = background_kind;
  for (int c = 0; c < 3; ++c) {
    s->env_down[c] = down ? down[c] : 0.f;
    s->env_up[c] = up ? up[c] : 0.f;
  }
  return 0;
}

int mref_scene_set_render_parameters(void* h, int max_depth, float cutoff) {
  RefScene* s = static_cast<RefScene*>(h);
  if (!s->scene) s->scene = new Scene();
  s->scene->getRenderParameters().maxDepth = max_depth;
  s->scene->getRenderParameters().importanceCutoff = cutoff;
  return 0;
}

// Makes material k of a scene a Phong (Model/Materials/Phong.cc) with the
// material's diffuse colour, the given specular colour, exponent and
// reflectivity (0: no reflection), in place of its Lambertian.
int mref_scene_set_phong(void* h, int k, const float* specular, int specpow, float refl) {
  RefScene* s = static_cast<RefScene*>(h);
  if (!s->mesh || k < 0 || k >= (int)s->mesh->materials.size()) return 1;
  Material* old = s->mesh->materials[k];
  Lambertian* lam = dynamic_cast<Lambertian*>(old);
  if (!lam) return 2;
  const float* kd = s->diffuse.data() + 3 * k;
  Material* ph = new Phong(Color(RGB(kd[0], kd[1], kd[2])),
                           Color(RGB(specular[0], specular[1], specular[2])), specpow, refl);
  s->mesh->materials[k] = ph;
  for (size_t i = 0; i < s->materials.size(); ++i)
    if (s->materials[i] == old) s->materials[i] = ph;
  return 0;
}

// Moves the mesh's vertices and refits the way the reference does for an
// animated mesh: WaldTriangle::update on every triangle (WaldTriangle.cc:
// 17-25; Kensler-Shirley triangles read the mesh directly), then
// DynBVH::update (DynBVH.cc:1574-1581).
int mref_scene_update_vertices(void* h, const float* verts, int nverts) {
  RefScene* s = static_cast<RefScene*>(h);
  if (!s->mesh || nverts != (int)s->mesh->vertices.size()) return 1;
  for (int i = 0; i < nverts; ++i)
    s->mesh->vertices[i] = Vector(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
  for (size_t t = 0; t < s->mesh->size(); ++t) {
    WaldTriangle* w = dynamic_cast<WaldTriangle*>(s->mesh->get(t));
    if (w) w->update();
  }
  s->bvh->update(0, 1);
#ifdef MREF_DROPIN
  // a scene rendering through the drop-in updates that tree as well
  if (GpuDynBVH* g = dynamic_cast<GpuDynBVH*>(s->object)) g->update(0, 1);
#endif
  return 0;
}

// Manta::readPlyFile (Model/Readers/PlyReader.cc:135-269) into a fresh
// Mesh with the given 3x4 transform (NULL = identity).  Returns the counts
// and, when the arrays are given and large enough, the vertices, indices
// and face materials.  0 = ok, 1 = the reader failed, 2 = arrays too small.
int mref_read_ply(const char* path, const float* transform, int tri_kind, int* nv, int* nt,
                  float* verts, unsigned* idx, unsigned* fmat, int cap_v, int cap_t) {
  try {
    AffineTransform t;
    t.initWithIdentity();
    if (transform)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) t.mat[i][j] = transform[4 * i + j];
    Mesh* m = new Mesh();
    if (!readPlyFile(std::string(path), t, m, 0,
                     tri_kind == 0 ? MeshTriangle::WALD_TRI
                                   : MeshTriangle::KENSLER_SHIRLEY_TRI))
      return 1;
    *nv = (int)m->vertices.size();
    *nt = (int)(m->vertex_indices.size() / 3);
    if (!verts) return 0;
    if (*nv > cap_v || *nt > cap_t) return 2;
    for (int i = 0; i < *nv; ++i)
      for (int c = 0; c < 3; ++c) verts[3 * i + c] = m->vertices[i][c];
    for (int i = 0; i < 3 * *nt; ++i) idx[i] = m->vertex_indices[i];
    for (int i = 0; i < *nt; ++i) fmat[i] = m->face_material[i];
    return 0;
  } catch (...) {
    return 1;
  }
}

// Manta::ObjGroup (Model/Groups/ObjGroup.cc:176-320) reading an OBJ file:
// counts, and when the arrays are large enough the vertices, triangles, face
// materials and, per entry of ObjGroup's material table, the kind of
// material it made (0 Lambertian, 1 Phong, 2 Dielectric, 3 Transparent,
// 4 for entry 0, ObjGroup's default) with the glm material values it was
// made from (diffuse rgb, specular rgb, Ns, Ni, d, filter rgb,
// reflectivity; glm_reader's model, read once more with glmReadOBJ).
// 0 = ok, 1 = the reader failed, 2 = arrays too small.
int mref_read_obj(const char* path, int tri_kind, int* nv, int* nt, int* nm, float* verts,
                  unsigned* idx, unsigned* fmat, int* kind, float* mvals, int cap_v,
                  int cap_t, int cap_m) {
  ObjGroup* g = 0;
  try {
    g = new ObjGroup(path, NULL, tri_kind == 0 ? MeshTriangle::WALD_TRI
                                                : MeshTriangle::KENSLER_SHIRLEY_TRI);
  } catch (...) {
    return 1;
  }
  *nv = (int)g->vertices.size();
  *nt = (int)(g->vertex_indices.size() / 3);
  *nm = (int)g->materials.size();
  if (!verts) return 0;
  if (*nv > cap_v || *nt > cap_t || *nm > cap_m) return 2;
  for (int i = 0; i < *nv; ++i)
    for (int c = 0; c < 3; ++c) verts[3 * i + c] = g->vertices[i][c];
  for (int i = 0; i < 3 * *nt; ++i) idx[i] = g->vertex_indices[i];
  for (int i = 0; i < *nt; ++i) fmat[i] = g->face_material[i];
  Glm::GLMmodel* model = Glm::glmReadOBJ(path);
  for (int i = 0; i < *nm; ++i) {
    const Material* m = g->materials[i];
    int k = 0;
    if (i == 0) k = 4;
    else if (dynamic_cast<const Dielectric*>(m)) k = 2;
    else if (dynamic_cast<const Transparent*>(m)) k = 3;
    else if (dynamic_cast<const Phong*>(m)) k = 1;
    else if (dynamic_cast<const Lambertian*>(m)) k = 0;
    else k = -1;
    kind[i] = k;
    float* q = mvals + 13 * i;
    for (int c = 0; c < 13; ++c) q[c] = 0;
    if (i > 0 && model && (unsigned)(i - 1) < model->nummaterials) {
      const Glm::GLMmaterial& gm = model->materials[i - 1];
      for (int c = 0; c < 3; ++c) {
        q[c] = gm.diffuse[c];
        q[3 + c] = gm.specular[c];
        q[9 + c] = gm.filter[c];
      }
      q[6] = gm.shininess;
      q[7] = gm.refraction;
      q[8] = gm.alpha;
      q[12] = gm.reflectivity;
    }
  }
  if (model) Glm::glmDelete(model);
  return 0;
}

void mref_scene_destroy(void* h) {
  // The reference never frees scene objects (Scene/Mesh own raw pointers);
  // only the harness record is released.
  delete static_cast<RefScene*>(h);
}

// Number of nodes the builder used (reachable from the root), the size of
// the node vector saveToFile writes, and the object_ids count.
int mref_tree_count(void* h, int* nodes_used, int* nodes_alloc, int* nids) {
  RefScene* s = static_cast<RefScene*>(h);
  const std::vector<DynBVH::BVHNode>& n = s->bvh->treeNodes();
  int maxIdx = 0;
  std::vector<int> stack(1, 0);
  while (!stack.empty()) {
    int i = stack.back();
    stack.pop_back();
    if (i > maxIdx) maxIdx = i;
    if (!n[i].isLeaf()) {
      stack.push_back(n[i].child);
      stack.push_back(n[i].child + 1);
    }
  }
  *nodes_used = maxIdx + 1;
  *nodes_alloc = (int)n.size();
  *nids = (int)s->bvh->treeIds().size();
  return 0;
}

// Field-wise export of the first nodes_used nodes plus object_ids.
int mref_tree_export(void* h, int nodes_used, float* bounds, int* child,
                     int* children, unsigned char* axis,
                     unsigned char* left_cheaper, int* ids) {
  RefScene* s = static_cast<RefScene*>(h);
  const std::vector<DynBVH::BVHNode>& n = s->bvh->treeNodes();
  for (int i = 0; i < nodes_used; ++i) {
    for (int c = 0; c < 3; ++c) {
      bounds[6 * i + c] = n[i].bounds[0][c];
      bounds[6 * i + 3 + c] = n[i].bounds[1][c];
    }
    child[i] = n[i].child;
    children[i] = n[i].children;
    axis[i] = n[i].axis;
    left_cheaper[i] = n[i].isLeftCheaper;
  }
  const std::vector<int>& o = s->bvh->treeIds();
  for (size_t i = 0; i < o.size(); ++i) ids[i] = o[i];
  return 0;
}

// The first n per-node costs (n <= the node vector's size) and nextFree.
int mref_tree_state(void* h, float* costs, int n, int* next_free) {
  RefScene* s = static_cast<RefScene*>(h);
  const std::vector<Real>& c = s->bvh->treeCosts();
  if (n > (int)c.size()) return 1;
  for (int i = 0; i < n; ++i) costs[i] = c[i];
  *next_free = s->bvh->nextFreeNode();
  return 0;
}

// DynBVH::saveToFile (DynBVH.cc:2479-2501) byte stream.
int mref_tree_save(void* h, const char* path) {
  RefScene* s = static_cast<RefScene*>(h);
  return s->bvh->saveToFile(std::string(path)) ? 0 : 1;
}

// sizeof(DynBVH::BVHNode) as compiled here (the saveToFile record size).
int mref_node_size() { return (int)sizeof(DynBVH::BVHNode); }

double mref_tree_cost(void* h) {
  return static_cast<RefScene*>(h)->bvh->sahCost();
}

// DynBVH::intersect over packets of `packet` consecutive rays.  org/dir are
// SoA ([x0..xn-1, y0.., z0..]).  Per ray: hit flag, t, triangle id, scratch
// u/v (WaldTriangle lambda/mue, KS uoverd/voverd).  anyhit sets
// RayPacket::AnyHit (HardShadows.cc:79).
int mref_intersect2(void* h, int n, const float* org, const float* dir,
                    const float* tmax, int anyhit, int packet, int* hit,
                    float* t, int* prim, float* u, float* v, int* inst) {
  RefScene* s = static_cast<RefScene*>(h);
  if (packet < 1 || packet > RayPacket::MaxSize) packet = RayPacket::MaxSize;
  RenderContext ctx(0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0);
  for (int base = 0; base < n; base += packet) {
    int cnt = n - base < packet ? n - base : packet;
    RayPacketData data;
    RayPacket rays(data, RayPacket::UnknownShape, 0, cnt, 0,
                   anyhit ? RayPacket::AnyHit : 0);
    for (int i = 0; i < cnt; ++i) {
      int r = base + i;
      rays.setRay(i, Vector(org[r], org[n + r], org[2 * n + r]),
                  Vector(dir[r], dir[n + r], dir[2 * n + r]));
      rays.resetHit(i, tmax[r]);
    }
    s->object->intersect(ctx, rays);
    for (int i = 0; i < cnt; ++i) {
      int r = base + i;
      hit[r] = rays.wasHit(i) ? 1 : 0;
      t[r] = rays.getMinT(i);
      int k = -1;
      if (hit[r]) {
        prim[r] = hit_prim(s, rays, i, &k);
        // an InstanceT hit keeps the inner u/v in the instance's own packet
        u[r] = k < 0 ? rays.getScratchpad<Real>(WaldTriangle::SCRATCH_U)[i] : 0.f;
        v[r] = k < 0 ? rays.getScratchpad<Real>(WaldTriangle::SCRATCH_V)[i] : 0.f;
      } else {
        prim[r] = -1;
        u[r] = 0.f;
        v[r] = 0.f;
      }
      if (inst) inst[r] = k;
    }
  }
  return 0;
}

int mref_intersect(void* h, int n, const float* org, const float* dir,
                   const float* tmax, int anyhit, int packet, int* hit,
                   float* t, int* prim, float* u, float* v) {
  return mref_intersect2(h, n, org, dir, tmax, anyhit, packet, hit, t, prim, u, v, 0);
}

struct QueryJob {
  RefScene* s;
  int n, anyhit;
  const float *org, *dir, *tmax;
  int* hit;
  float* t;
  int* prim;
  volatile int next;
  pthread_mutex_t lock;
  int nthreads;
};

struct QueryArg {
  QueryJob* job;
  int proc;
};

static void* query_worker(void* p) {
  QueryArg* a = static_cast<QueryArg*>(p);
  QueryJob* j = a->job;
  RenderContext ctx(0, 0, a->proc, j->nthreads, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0);
  const int P = RayPacket::MaxSize;
  for (;;) {
    pthread_mutex_lock(&j->lock);
    const int base = j->next;
    j->next += 16 * P;
    pthread_mutex_unlock(&j->lock);
    if (base >= j->n) break;
    const int stop = base + 16 * P < j->n ? base + 16 * P : j->n;
    for (int b = base; b < stop; b += P) {
      const int cnt = stop - b < P ? stop - b : P;
      RayPacketData data;
      RayPacket rays(data, RayPacket::UnknownShape, 0, cnt, 0,
                     j->anyhit ? RayPacket::AnyHit : 0);
      const int n = j->n;
      for (int i = 0; i < cnt; ++i) {
        const int r = b + i;
        rays.setRay(i, Vector(j->org[r], j->org[n + r], j->org[2 * n + r]),
                    Vector(j->dir[r], j->dir[n + r], j->dir[2 * n + r]));
        rays.resetHit(i, j->tmax[r]);
      }
      j->s->object->intersect(ctx, rays);
      for (int i = 0; i < cnt; ++i) {
        const int r = b + i;
        j->hit[r] = rays.wasHit(i) ? 1 : 0;
        j->t[r] = rays.getMinT(i);
        j->prim[r] = j->hit[r] ? hit_prim(j->s, rays, i, 0) : -1;
      }
    }
  }
  return 0;
}

// DynBVH::intersect over 64-ray packets on N pthreads (packets taken 16 at a
// time from a shared counter).  Returns wall seconds in *seconds.
int mref_intersect_mt(void* h, int n, const float* org, const float* dir, const float* tmax,
                      int anyhit, int nthreads, int* hit, float* t, int* prim,
                      double* seconds) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  QueryJob job;
  job.s = static_cast<RefScene*>(h);
  job.n = n;
  job.anyhit = anyhit;
  job.org = org;
  job.dir = dir;
  job.tmax = tmax;
  job.hit = hit;
  job.t = t;
  job.prim = prim;
  job.next = 0;
  job.nthreads = nthreads;
  pthread_mutex_init(&job.lock, 0);
  std::vector<pthread_t> th(nthreads);
  std::vector<QueryArg> ar(nthreads);
  const double t0 = now_s();
  for (int p = 0; p < nthreads; ++p) {
    ar[p].job = &job;
    ar[p].proc = p;
    pthread_create(&th[p], 0, query_worker, &ar[p]);
  }
  for (int p = 0; p < nthreads; ++p) pthread_join(th[p], 0);
  const double t1 = now_s();
  pthread_mutex_destroy(&job.lock);
  if (seconds) *seconds = t1 - t0;
  return 0;
}

// Camera basis (eye, lookat-eye, u, v) of PinholeCamera with the given
// eye/lookat/up/hfov/vfov and -normalizeRays.
int mref_camera_basis(const float* eye, const float* lookat, const float* up,
                      float hfov, float vfov, float* out12) {
  char buf[16][32];
  std::vector<std::string> args;
  args.push_back("-eye");
  for (int i = 0; i < 3; ++i) { snprintf(buf[i], 32, "%.9g", eye[i]); args.push_back(buf[i]); }
  args.push_back("-lookat");
  for (int i = 0; i < 3; ++i) { snprintf(buf[3 + i], 32, "%.9g", lookat[i]); args.push_back(buf[3 + i]); }
  args.push_back("-up");
  for (int i = 0; i < 3; ++i) { snprintf(buf[6 + i], 32, "%.9g", up[i]); args.push_back(buf[6 + i]); }
  args.push_back("-hfov"); snprintf(buf[9], 32, "%.9g", hfov); args.push_back(buf[9]);
  args.push_back("-vfov"); snprintf(buf[10], 32, "%.9g", vfov); args.push_back(buf[10]);
  args.push_back("-normalizeRays");
  try {
    ExposedCamera cam(args);
    cam.basis(out12);
  } catch (Exception& e) {
    fprintf(stderr, "mref_camera_basis: %s\n", e.message());
    return 1;
  } catch (...) {
    return 1;
  }
  return 0;
}

struct RenderJob {
  RefScene* s;
  Raytracer* renderer;
  CountingShadows* shadows;
  ExposedCamera* camera;
  ConstantSampleGenerator* sampler;
  int xres, yres;
  float xscale, yscale, xoffset, yoffset;
  float* rgb;
  float* tprim;
  int* prim;
  volatile int next_row;
  pthread_mutex_t lock;
  long long shadow_rays[256];
  int nthreads;
};

struct RenderArg {
  RenderJob* job;
  int proc;
};

static void* render_worker(void* p) {
  RenderArg* a = static_cast<RenderArg*>(p);
  RenderJob* j = a->job;
  CountingShadows shadows;  // per-thread (it carries the counter slot)
  shadows.counter = &j->shadow_rays[a->proc];
  ShadowAlgorithm* sa = &shadows;
#ifdef MREF_DROPIN
  CountingGpuShadows* gpu_shadows = 0;
  if (j->s->gpu_shadows) {
    GpuDynBVH* g = dynamic_cast<GpuDynBVH*>(j->s->object);
    if (!g) {
      Group* grp = dynamic_cast<Group*>(j->s->object);
      GpuMeshPrimitive* p =
          grp && grp->size() > 0 ? dynamic_cast<GpuMeshPrimitive*>(grp->get(0)) : 0;
      g = p ? p->bvh() : 0;
    }
    gpu_shadows = new CountingGpuShadows(g);
    gpu_shadows->counter = &j->shadow_rays[a->proc];
    sa = gpu_shadows;
  }
#endif
  RenderContext ctx(0, 0, a->proc, j->nthreads, 0, 0, 0, j->renderer, sa,
                    j->camera, j->s->scene, 0, 0, j->sampler);
  for (;;) {
    pthread_mutex_lock(&j->lock);
    int y = j->next_row++;
    pthread_mutex_unlock(&j->lock);
    if (y >= j->yres) break;
    for (int x0 = 0; x0 < j->xres; x0 += RayPacket::MaxSize) {
      int cnt = j->xres - x0 < RayPacket::MaxSize ? j->xres - x0 : (int)RayPacket::MaxSize;
      RayPacketData data;
      RayPacket rays(data, RayPacket::UnknownShape, 0, cnt, 0,
                     RayPacket::HaveImageCoordinates | RayPacket::ConstantEye);
      for (int i = 0; i < cnt; ++i) {
        // Image coordinates per pixel in closed form (SingleSampler.cc:38-41
        // scale/offset); the reference's frame loop accumulates px instead.
        Real px = (Real)(x0 + i) * j->xscale + j->xoffset;
        Real py = (Real)y * j->yscale + j->yoffset;
        rays.setPixel(i, 0, px, py);
      }
      j->renderer->traceEyeRays(ctx, rays);
      for (int i = 0; i < cnt; ++i) {
        size_t pix = (size_t)y * j->xres + x0 + i;
        Color c = rays.getColor(i);
        j->rgb[3 * pix + 0] = c[0];
        j->rgb[3 * pix + 1] = c[1];
        j->rgb[3 * pix + 2] = c[2];
        if (j->prim) {
          bool h = rays.wasHit(i);
          j->prim[pix] = h ? hit_prim(j->s, rays, i, 0) : -1;
          j->tprim[pix] = rays.getMinT(i);
        }
      }
    }
  }
#ifdef MREF_DROPIN
  delete gpu_shadows;
#endif
  return 0;
}

// Whitted frame through Raytracer::traceEyeRays.  lights: nlights x
// (px,py,pz, r,g,b).  ambient/background: RGB.  Returns wall seconds of the
// frame loop in *seconds and the shadow-ray count in *shadow_rays.
int mref_render(void* h, int xres, int yres, const float* cam12_args,
                const float* lights, int nlights, const float* ambient,
                const float* background, int nthreads, float* rgb,
                float* tprim, int* prim, double* seconds,
                long long* shadow_rays) {
  RefScene* s = static_cast<RefScene*>(h);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  // cam12_args: eye[3], lookat[3], up[3], hfov, vfov, unused
  char buf[16][32];
  std::vector<std::string> args;
  const char* names[3] = {"-eye", "-lookat", "-up"};
  for (int k = 0; k < 3; ++k) {
    args.push_back(names[k]);
    for (int i = 0; i < 3; ++i) {
      snprintf(buf[3 * k + i], 32, "%.9g", cam12_args[3 * k + i]);
      args.push_back(buf[3 * k + i]);
    }
  }
  args.push_back("-hfov"); snprintf(buf[9], 32, "%.9g", cam12_args[9]); args.push_back(buf[9]);
  args.push_back("-vfov"); snprintf(buf[10], 32, "%.9g", cam12_args[10]); args.push_back(buf[10]);
  args.push_back("-normalizeRays");
  ExposedCamera camera(args);

  LightSet* ls = new LightSet();
  ls->setAmbientLight(make_ambient(s, ambient));
  for (int k = 0; k < nlights; ++k) {
    const float* L = lights + 6 * k;
    ls->add(new PointLight(Vector(L[0], L[1], L[2]), Color(RGB(L[3], L[4], L[5]))));
  }
  PreprocessContext pctx;
  pctx.globalLights = ls;
  for (size_t k = 0; k < s->materials.size(); ++k) s->materials[k]->preprocess(pctx);
  if (!s->scene) s->scene = new Scene();
  s->scene->setObject(s->object);
  s->scene->setBackground(make_background(s, background));
  s->scene->setLights(ls);

  Raytracer renderer;
  ConstantSampleGenerator sampler(0.f);
  RenderJob job;
  job.s = s;
  job.renderer = &renderer;
  job.camera = &camera;
  job.sampler = &sampler;
  job.xres = xres;
  job.yres = yres;
  job.xscale = (Real)2 / xres;
  job.yscale = (Real)2 / yres;
  job.xoffset = (-xres / (Real)2 + (Real)0.5) * job.xscale;
  job.yoffset = (-yres / (Real)2 + (Real)0.5) * job.yscale;
  job.rgb = rgb;
  job.tprim = tprim;
  job.prim = prim;
  job.next_row = 0;
  job.nthreads = nthreads;
  memset(job.shadow_rays, 0, sizeof(job.shadow_rays));
  pthread_mutex_init(&job.lock, 0);
  std::vector<pthread_t> th(nthreads);
  std::vector<RenderArg> ar(nthreads);
  double t0 = now_s();
  for (int p = 0; p < nthreads; ++p) {
    ar[p].job = &job;
    ar[p].proc = p;
    pthread_create(&th[p], 0, render_worker, &ar[p]);
  }
  for (int p = 0; p < nthreads; ++p) pthread_join(th[p], 0);
  double t1 = now_s();
  pthread_mutex_destroy(&job.lock);
  long long total = 0;
  for (int p = 0; p < nthreads; ++p) total += job.shadow_rays[p];
  if (seconds) *seconds = t1 - t0;
  if (shadow_rays) *shadow_rays = total;
  return 0;
}

// Two-level scene: per instance the inner scene's DynBVH wrapped in an
// InstanceT (kind 0, Model/Instances/InstanceT.cc; called through
// InstanceGuard) or placed in the top-level Group itself (kind 1); a
// top-level DynBVH is built over the Group.  Inner scenes come from
// mref_scene_create and must outlive it.
void* mref_scene_create_instanced(void* const* inner, int n_inner, const int* inst_scene,
                                  const float* inst_T, const int* inst_kind, int n_inst) {
  try {
    RefScene* s = new RefScene();
    s->mesh = 0;
    s->scene = 0;
    Group* g = new Group();
    for (int k = 0; k < n_inst; ++k) {
      if (inst_scene[k] < 0 || inst_scene[k] >= n_inner) return 0;
      RefScene* b = static_cast<RefScene*>(inner[inst_scene[k]]);
      const int kind = inst_kind ? inst_kind[k] : 0;
      if (kind == 0) {
        InstanceT* it = new InstanceT(
            b->bvh, Vector(inst_T[3 * k], inst_T[3 * k + 1], inst_T[3 * k + 2]));
        s->instance_of[it] = k;
        g->add(new InstanceGuard(it));
      } else {
        g->add(b->bvh);
      }
    }
    for (int i = 0; i < n_inner; ++i) {
      RefScene* b = static_cast<RefScene*>(inner[i]);
      s->materials.insert(s->materials.end(), b->materials.begin(), b->materials.end());
    }
    s->lights = new LightSet();
    s->lights->setAmbientLight(new ConstantAmbient(Color(RGB(0, 0, 0))));
    s->bvh = new ExposedBVH();
    s->bvh->setGroup(g);
    s->bvh->rebuild(0, 1);
    s->object = s->bvh;
    return s;
  } catch (...) {
    return 0;
  }
}

struct CoordJob {
  RefScene* s;
  Raytracer* renderer;
  ExposedCamera* camera;
  ConstantSampleGenerator* sampler;
  int n;
  const float* px;
  const float* py;
  float* rgb;
  float* tprim;
  int* prim;
  volatile int next;
  pthread_mutex_t lock;
  long long shadow_rays[256];
  int nthreads;
};

struct CoordArg {
  CoordJob* job;
  int proc;
};

static void* coord_worker(void* p) {
  CoordArg* a = static_cast<CoordArg*>(p);
  CoordJob* j = a->job;
  CountingShadows shadows;
  shadows.counter = &j->shadow_rays[a->proc];
  RenderContext ctx(0, 0, a->proc, j->nthreads, 0, 0, 0, j->renderer, &shadows,
                    j->camera, j->s->scene, 0, 0, j->sampler);
  const int P = RayPacket::MaxSize;
  for (;;) {
    pthread_mutex_lock(&j->lock);
    const int base = j->next;
    j->next += P;
    pthread_mutex_unlock(&j->lock);
    if (base >= j->n) break;
    const int cnt = j->n - base < P ? j->n - base : P;
    RayPacketData data;
    RayPacket rays(data, RayPacket::UnknownShape, 0, cnt, 0,
                   RayPacket::HaveImageCoordinates | RayPacket::ConstantEye);
    for (int i = 0; i < cnt; ++i) rays.setPixel(i, 0, j->px[base + i], j->py[base + i]);
    j->renderer->traceEyeRays(ctx, rays);
    for (int i = 0; i < cnt; ++i) {
      const size_t r = (size_t)base + i;
      Color c = rays.getColor(i);
      for (int k = 0; k < 3; ++k) j->rgb[3 * r + k] = c[k];
      if (j->prim) {
        j->prim[r] = rays.wasHit(i) ? hit_prim(j->s, rays, i, 0) : -1;
        j->tprim[r] = rays.getMinT(i);
      }
    }
  }
  return 0;
}

// Raytracer::traceEyeRays (as mref_render) for n eye rays at the given image
// coordinates, in packets of 64 consecutive rays on N pthreads.
int mref_render_coords(void* h, int n, const float* px, const float* py,
                       const float* cam12_args, const float* lights, int nlights,
                       const float* ambient, const float* background, int nthreads,
                       float* rgb, float* tprim, int* prim, long long* shadow_rays) {
  RefScene* s = static_cast<RefScene*>(h);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  char buf[16][32];
  std::vector<std::string> args;
  const char* names[3] = {"-eye", "-lookat", "-up"};
  for (int k = 0; k < 3; ++k) {
    args.push_back(names[k]);
    for (int i = 0; i < 3; ++i) {
      snprintf(buf[3 * k + i], 32, "%.9g", cam12_args[3 * k + i]);
      args.push_back(buf[3 * k + i]);
    }
  }
  args.push_back("-hfov"); snprintf(buf[9], 32, "%.9g", cam12_args[9]); args.push_back(buf[9]);
  args.push_back("-vfov"); snprintf(buf[10], 32, "%.9g", cam12_args[10]); args.push_back(buf[10]);
  args.push_back("-normalizeRays");
  ExposedCamera camera(args);
  LightSet* ls = new LightSet();
  ls->setAmbientLight(make_ambient(s, ambient));
  for (int k = 0; k < nlights; ++k) {
    const float* L = lights + 6 * k;
    ls->add(new PointLight(Vector(L[0], L[1], L[2]), Color(RGB(L[3], L[4], L[5]))));
  }
  PreprocessContext pctx;
  pctx.globalLights = ls;
  for (size_t k = 0; k < s->materials.size(); ++k) s->materials[k]->preprocess(pctx);
  if (!s->scene) s->scene = new Scene();
  s->scene->setObject(s->object);
  s->scene->setBackground(make_background(s, background));
  s->scene->setLights(ls);
  Raytracer renderer;
  ConstantSampleGenerator sampler(0.f);
  CoordJob job;
  job.s = s;
  job.renderer = &renderer;
  job.camera = &camera;
  job.sampler = &sampler;
  job.n = n;
  job.px = px;
  job.py = py;
  job.rgb = rgb;
  job.tprim = tprim;
  job.prim = prim;
  job.next = 0;
  job.nthreads = nthreads;
  memset(job.shadow_rays, 0, sizeof(job.shadow_rays));
  pthread_mutex_init(&job.lock, 0);
  std::vector<pthread_t> th(nthreads);
  std::vector<CoordArg> ar(nthreads);
  for (int p = 0; p < nthreads; ++p) {
    ar[p].job = &job;
    ar[p].proc = p;
    pthread_create(&th[p], 0, coord_worker, &ar[p]);
  }
  for (int p = 0; p < nthreads; ++p) pthread_join(th[p], 0);
  pthread_mutex_destroy(&job.lock);
  long long total = 0;
  for (int p = 0; p < nthreads; ++p) total += job.shadow_rays[p];
  if (shadow_rays) *shadow_rays = total;
  return 0;
}

struct PathJob {
  RefScene* s;
  KajiyaPathtracer* renderer;
  ExposedCamera* camera;
  int xres, yres, spp;
  float xscale, yscale, xoff, yoff;
  float* rgb;
  volatile int next_row;
  pthread_mutex_t lock;
  int nthreads;
  unsigned seed;
};

struct PathArg {
  PathJob* job;
  int proc;
};

static void* path_worker(void* p) {
  PathArg* a = static_cast<PathArg*>(p);
  PathJob* j = a->job;
  HardShadows shadows(false);
  CheapRNG rng;
  rng.seed(j->seed + 7919u * (unsigned)a->proc);
  UniformRandomGenerator sampler;
  RenderContext ctx(0, 0, a->proc, j->nthreads, 0, 0, 0, j->renderer, &shadows, j->camera,
                    j->s->scene, 0, &rng, &sampler);
  int strata = 1;
  while (strata * strata < j->spp) ++strata;
  for (;;) {
    pthread_mutex_lock(&j->lock);
    int y = j->next_row++;
    pthread_mutex_unlock(&j->lock);
    if (y >= j->yres) break;
    for (int x0 = 0; x0 < j->xres; x0 += RayPacket::MaxSize) {
      int cnt = j->xres - x0 < RayPacket::MaxSize ? j->xres - x0 : (int)RayPacket::MaxSize;
      float acc[3][RayPacket::MaxSize];
      memset(acc, 0, sizeof(acc));
      for (int sidx = 0; sidx < j->spp; ++sidx) {
        RayPacketData data;
        RayPacket rays(data, RayPacket::UnknownShape, 0, cnt, 0,
                       RayPacket::HaveImageCoordinates | RayPacket::ConstantEye);
        const int sx = sidx % strata, sy = sidx / strata;
        for (int i = 0; i < cnt; ++i) {
          // stratified jitter inside the pixel
          float jx = j->spp > 1 ? (sx + rng.nextFloat()) / strata : 0.5f;
          float jy = j->spp > 1 ? (sy + rng.nextFloat()) / strata : 0.5f;
          rays.setPixel(i, 0, (x0 + i + jx) * j->xscale + j->xoff, (y + jy) * j->yscale + j->yoff);
        }
        j->renderer->traceEyeRays(ctx, rays);
        for (int i = 0; i < cnt; ++i) {
          Color c = rays.getColor(i);
          for (int k = 0; k < 3; ++k) acc[k][i] += c[k];
        }
      }
      for (int i = 0; i < cnt; ++i) {
        size_t pix = (size_t)y * j->xres + x0 + i;
        for (int k = 0; k < 3; ++k) j->rgb[3 * pix + k] = acc[k][i] / j->spp;
      }
    }
  }
  return 0;
}

// Path-traced frame through KajiyaPathtracer::traceEyeRays
// (Engine/Renderers/KajiyaPathtracer.cc:113-302) with its default modes,
// HardShadows, one Parallelogram AreaLight and a ConstantAmbient
// (background[0..2] then the ambient colour in background[3..5]); rows of
// 64-ray packets on N
// pthreads, spp stratified-jitter packets per pixel row segment.  *rays =
// every unmasked ray handed to DynBVH::intersect (camera, bounce, shadow).
int mref_render_path(void* h, int xres, int yres, const float* cam11, int spp,
                     int max_depth, const float* light12, const float* background,
                     int nthreads, unsigned seed, float* rgb, double* seconds,
                     long long* rays) {
  RefScene* s = static_cast<RefScene*>(h);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  char buf[16][32];
  std::vector<std::string> args;
  const char* names[3] = {"-eye", "-lookat", "-up"};
  for (int k = 0; k < 3; ++k) {
    args.push_back(names[k]);
    for (int i = 0; i < 3; ++i) {
      snprintf(buf[3 * k + i], 32, "%.9g", cam11[3 * k + i]);
      args.push_back(buf[3 * k + i]);
    }
  }
  args.push_back("-hfov"); snprintf(buf[9], 32, "%.9g", cam11[9]); args.push_back(buf[9]);
  args.push_back("-vfov"); snprintf(buf[10], 32, "%.9g", cam11[10]); args.push_back(buf[10]);
  args.push_back("-normalizeRays");
  ExposedCamera camera(args);
  LightSet* ls = new LightSet();
  ls->setAmbientLight(make_ambient(s, background + 3));
  Parallelogram* emitter = new Parallelogram(s->materials[0],
      Vector(light12[0], light12[1], light12[2]), Vector(light12[3], light12[4], light12[5]),
      Vector(light12[6], light12[7], light12[8]));
  ls->add(new AreaLight(emitter, Color(RGB(light12[9], light12[10], light12[11]))));
  PreprocessContext pctx;
  pctx.globalLights = ls;
  for (size_t k = 0; k < s->materials.size(); ++k) s->materials[k]->preprocess(pctx);
  if (!s->scene) s->scene = new Scene();
  s->scene->setObject(s->object);
  s->scene->setBackground(make_background(s, background));
  s->scene->setLights(ls);
  s->scene->getRenderParameters().maxDepth = max_depth;
  std::vector<std::string> none;
  KajiyaPathtracer renderer(none);
  std::vector<long long> counters(16 * nthreads, 0);
  s->bvh->ray_counters = &counters[0];
  PathJob job;
  job.s = s;
  job.renderer = &renderer;
  job.camera = &camera;
  job.xres = xres;
  job.yres = yres;
  job.spp = spp;
  job.xscale = (Real)2 / xres;
  job.yscale = (Real)2 / yres;
  job.xoff = (-xres / (Real)2) * job.xscale;
  job.yoff = (-yres / (Real)2) * job.yscale;
  job.rgb = rgb;
  job.next_row = 0;
  job.nthreads = nthreads;
  job.seed = seed;
  pthread_mutex_init(&job.lock, 0);
  std::vector<pthread_t> th(nthreads);
  std::vector<PathArg> ar(nthreads);
  double t0 = now_s();
  for (int p = 0; p < nthreads; ++p) {
    ar[p].job = &job;
    ar[p].proc = p;
    pthread_create(&th[p], 0, path_worker, &ar[p]);
  }
  for (int p = 0; p < nthreads; ++p) pthread_join(th[p], 0);
  double t1 = now_s();
  pthread_mutex_destroy(&job.lock);
  s->bvh->ray_counters = 0;
  long long total = 0;
  for (int p = 0; p < nthreads; ++p) total += counters[16 * p];
  if (seconds) *seconds = t1 - t0;
  if (rays) *rays = total;
  return 0;
}

#ifdef MREF_DROPIN
// Swaps the scene's DynBVH for the GPU drop-in (rfmanta_b200/manta/
// GpuDynBVH), so the reference's own Raytracer, Lambertian and HardShadows
// run unchanged on top of it.  tree_file NULL: the drop-in builds its own
// tree (GpuDynBVH::rebuild); else the reference tree is written there with
// DynBVH::saveToFile and read back with GpuDynBVH::buildFromFile.
int mref_scene_use_gpu(void* h, int device, int tri_kind, const char* tree_file) {
  RefScene* s = static_cast<RefScene*>(h);
  try {
    GpuDynBVH* g = new GpuDynBVH(device, tri_kind);
    g->setGroup(s->mesh);
    if (tree_file) {
      if (!s->bvh->saveToFile(std::string(tree_file))) return 2;
      if (!g->buildFromFile(std::string(tree_file))) return 3;
    } else {
      g->rebuild(0, 1);
    }
    s->object = g;
  } catch (Exception& e) {
    fprintf(stderr, "mref_scene_use_gpu: %s\n", e.message());
    return 1;
  }
  return 0;
}

// Options of a scene already swapped to the drop-in: how packets reach the
// device (GpuDynBVH::setPacketMode: 0 one round trip per call, 1 the
// submission queue, 2 the resident packet channel), and
// GpuHardShadows for Whitted renders.
int mref_scene_gpu_options(void* h, int batching, int gpu_shadows) {
  RefScene* s = static_cast<RefScene*>(h);
  GpuDynBVH* g = dynamic_cast<GpuDynBVH*>(s->object);
  if (!g) {
    Group* grp = dynamic_cast<Group*>(s->object);
    GpuMeshPrimitive* p =
        grp && grp->size() > 0 ? dynamic_cast<GpuMeshPrimitive*>(grp->get(0)) : 0;
    g = p ? p->bvh() : 0;
  }
  if (!g) return 1;
  g->setPacketMode(batching);
  s->gpu_shadows = gpu_shadows;
  return 0;
}

// The drop-in as a Primitive: the scene's object becomes a reference Group
// holding one GpuMeshPrimitive over the scene's GpuDynBVH (after
// mref_scene_use_gpu), traced through Group::intersect.
int mref_scene_gpu_as_primitive(void* h) {
  RefScene* s = static_cast<RefScene*>(h);
  GpuDynBVH* g = dynamic_cast<GpuDynBVH*>(s->object);
  if (!g) return 1;
  Group* grp = new Group();
  grp->add(new GpuMeshPrimitive(g));
  s->object = grp;
  return 0;
}
#endif

}  // extern "C"
