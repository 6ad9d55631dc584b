// GpuDynBVH: see GpuDynBVH.h.
#include "GpuDynBVH.h"

#include <Core/Color/Color.h>
#include <Core/Exceptions/InternalError.h>
#include <Core/Geometry/BBox.h>
#include <Interface/Context.h>
#include <Interface/Material.h>
#include <Interface/TexCoordMapper.h>
#include <Model/Groups/Mesh.h>
#include <Model/Primitives/MeshTriangle.h>
#include <Model/Primitives/WaldTriangle.h>

#include <fstream>
#include <vector>

using namespace Manta;

// Rays per batch of the submission queue: 256 packets of 64 rays.
static const int kQueueRays = 256 * RayPacket::MaxSize;

GpuDynBVH::GpuDynBVH(int device_, int tri_kind_)
    : group(0), mesh(0), scene(0), queue(0), channel(0), device(device_), tri_kind(tri_kind_),
      dirty(false), mode(Resident) {}

GpuDynBVH::~GpuDynBVH() {
  if (channel) rq_channel_destroy(channel);
  if (queue) rq_queue_destroy(queue);
  if (scene) rq_scene_destroy(scene);
}

void GpuDynBVH::setPacketMode(int m) {
  if (m != PerCall && m != Queue && m != Resident)
    throw InternalError("GpuDynBVH::setPacketMode: PerCall, Queue or Resident");
  mode = m;
  // an idle channel's kernel is stopped at once rather than at its idle limit
  if (mode != Resident && channel) rq_channel_stop(channel);
}

void GpuDynBVH::setBatching(bool on) { setPacketMode(on ? Queue : PerCall); }

void GpuDynBVH::check(int rc, const char* what) const {
  if (rc != RQ_OK)
    throw InternalError(std::string("rfmanta_b200 ") + what + ": " + rq_last_error());
}

void GpuDynBVH::setGroup(Group* g) {
  if (g != group) dirty = true;
  group = g;
  mesh = dynamic_cast<Mesh*>(g);
}

void GpuDynBVH::groupDirty() { dirty = true; }

Group* GpuDynBVH::getGroup() const { return group; }

void GpuDynBVH::addToUpdateGraph(ObjectUpdateGraph* graph, ObjectUpdateGraphNode* parent) {
  (void)graph;
  (void)parent;
}

Interpolable::InterpErr GpuDynBVH::parallelInterpolate(const std::vector<keyframe_t>& keyframes, int proc,
                                         int numProc) {
  return group->parallelInterpolate(keyframes, proc, numProc);
}

// Mesh::vertices / vertex_indices / face_material (Model/Groups/Mesh.h:27-50).
void GpuDynBVH::upload() {
  if (!mesh) throw InternalError("GpuDynBVH needs a Mesh group");
  if (channel) {
    rq_channel_destroy(channel);
    channel = 0;
  }
  if (queue) {
    rq_queue_destroy(queue);
    queue = 0;
  }
  if (scene) {
    rq_scene_destroy(scene);
    scene = 0;
  }
  const size_t nv = mesh->vertices.size();
  std::vector<float> v(3 * nv);
  for (size_t i = 0; i < nv; ++i)
    for (int c = 0; c < 3; ++c) v[3 * i + c] = mesh->vertices[i][c];
  const int nt = (int)(mesh->vertex_indices.size() / 3);
  texmap.resize(mesh->size());
  for (size_t i = 0; i < texmap.size(); ++i)
    texmap[i] = dynamic_cast<const TexCoordMapper*>(mesh->get(i));
  check(rq_scene_create(&v[0], (int)nv, &mesh->vertex_indices[0], nt,
                        mesh->face_material.empty() ? 0 : &mesh->face_material[0], tri_kind,
                        device, &scene),
        "scene upload");
  check(rq_queue_create(scene, kQueueRays, &queue), "submission queue");
  // 128 slots: one per render worker up to 128 at a time (workers may
  // outnumber the cores, so some shade while others wait); 1024-ray packets
  // hold GpuHardShadows' shadow packets of up to 16 lights (larger ones take
  // the per-call path)
  check(rq_channel_create(scene, 128, 16 * RayPacket::MaxSize, &channel), "packet channel");
  dirty = false;
}

void GpuDynBVH::preprocess(const PreprocessContext& context) {
  if (group) group->preprocess(context);
  if (context.proc == 0 && (dirty || !scene)) rebuild(0, 1);
  context.done();
}

void GpuDynBVH::rebuild(int proc, int numProcs) {
  (void)numProcs;
  if (proc != 0) return;
  upload();
  check(rq_scene_build(scene, 0), "build");
}

// DynBVH::update (DynBVH.cc:1574-1581): the mesh moved; the device refits
// the tree and applies the reference's leaf re-splits and tree rotations
// (TREE_ROT 1, rotateNode DynBVH.cc:3051-3348).
void GpuDynBVH::update(int proc, int numProcs) {
  (void)numProcs;
  if (proc != 0) return;
  if (dirty || !scene) {
    rebuild(0, 1);
    return;
  }
  const size_t nv = mesh->vertices.size();
  std::vector<float> v(3 * nv);
  for (size_t i = 0; i < nv; ++i)
    for (int c = 0; c < 3; ++c) v[3 * i + c] = mesh->vertices[i][c];
  check(rq_scene_update_vertices_ex(scene, v.empty() ? 0 : &v[0], (int)nv, RQ_UPDATE_ROTATE),
        "update");
}

bool GpuDynBVH::buildFromFile(const std::string& file) {
  std::ifstream in(file.c_str(), std::ios::binary);
  if (!in) return false;
  std::vector<char> blob((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  upload();
  check(rq_scene_import_dynbvh(scene, blob.empty() ? 0 : &blob[0], blob.size()), "import");
  return true;
}

bool GpuDynBVH::saveToFile(const std::string& file) {
  if (!scene) return false;
  size_t n = 0;
  check(rq_scene_export_dynbvh(scene, 0, &n), "export");
  std::vector<char> blob(n);
  check(rq_scene_export_dynbvh(scene, &blob[0], &n), "export");
  std::ofstream out(file.c_str(), std::ios::binary);
  if (!out) return false;
  out.write(&blob[0], (std::streamsize)n);
  return true;
}

void GpuDynBVH::computeBounds(const PreprocessContext& context, BBox& bbox) const {
  group->computeBounds(context, bbox);
}

int GpuDynBVH::selectRays(const RayPacket& rays, bool any, int* map) const {
  int n = 0;
  for (int i = rays.begin(); i < rays.end(); ++i) {
    if (rays.rayIsMasked(i)) continue;
    if (any && rays.wasHit(i)) continue;
    map[n++] = i;
  }
  return n;
}

void GpuDynBVH::packRays(const RayPacket& rays, const int* map, int n, int stride, int base,
                         float* org, float* dir, float* tmax) {
  for (int k = 0; k < n; ++k) {
    const int i = map[k];
    for (int c = 0; c < 3; ++c) {
      org[c * stride + base + k] = rays.getOrigin(i, c);
      dir[c * stride + base + k] = rays.getDirection(i, c);
    }
    tmax[base + k] = rays.getMinT(i);
  }
}

void GpuDynBVH::traceRays(int n, const float* org, const float* dir, const float* tmax, bool any,
                          float* t, int* prim, float* u, float* v) const {
  const int flags = any ? RQ_ANYHIT : RQ_CLOSEST;
  if (mode == Resident && channel)
    check(rq_channel_trace(channel, n, org, dir, tmax, flags, t, prim, u, v), "channel trace");
  else if (mode == Queue && queue)
    check(rq_queue_trace(queue, n, org, dir, tmax, flags, t, prim, u, v), "queued trace");
  else
    check(rq_trace(scene, n, org, dir, tmax, flags, t, prim, u, v), "trace");
}

void GpuDynBVH::applyHits(const RenderContext& context, RayPacket& rays, bool any,
                          const int* map, int n, const float* t, const int* prim,
                          const float* u, const float* v) const {
  Real oldT[RayPacket::MaxSize];
  bool hit[RayPacket::MaxSize];
  for (int k = 0; k < n; ++k) {
    hit[k] = false;
    if (prim[k] < 0) continue;
    const int i = map[k];
    const MeshTriangle* tri = mesh->get(prim[k]);
    const Material* matl = mesh->materials[mesh->face_material[prim[k]]];
    const TexCoordMapper* tex = (size_t)prim[k] < texmap.size()
                                    ? texmap[prim[k]]
                                    : dynamic_cast<const TexCoordMapper*>(tri);
    oldT[k] = rays.getMinT(i);
    if (rays.hit(i, t[k], matl, tri, tex)) {
      hit[k] = true;
      rays.getScratchpad<Real>(WaldTriangle::SCRATCH_U)[i] = u[k];
      rays.getScratchpad<Real>(WaldTriangle::SCRATCH_V)[i] = v[k];
    }
  }
  if (!any) return;
  // occluded rays: the material attenuates them, over runs of adjacent rays
  // with the same hit material as DynBVH does (DynBVH.cc:320-345); an
  // attenuated ray is released again, an opaque one keeps its hit with
  // minT = T_EPSILON
  for (int k = 0; k < n; ++k) {
    if (!hit[k]) continue;
    const int i = map[k];
    const Material* matl = rays.getHitMaterial(i);
    int e = k + 1;
    while (e < n && hit[e] && map[e] == map[e - 1] + 1 && rays.getHitMaterial(map[e]) == matl)
      ++e;
    RayPacket run(rays, i, map[e - 1] + 1);
    matl->attenuateShadows(context, run);
    for (int q = k; q < e; ++q) {
      if (run.getColor(map[q]) != Color::black())
        rays.resetHit(map[q], oldT[q]);
      else
        rays.overrideMinT(map[q], T_EPSILON);
    }
    k = e - 1;
  }
}

// DynBVH::intersect (Model/Groups/DynBVH.cc:101-404) for one packet: the
// unmasked (and, for AnyHit, not yet hit) rays go to the device; hits come
// back through RayPacket::hit with the real MeshTriangle, its material and
// the scratchpad pair; occluded AnyHit rays are then treated as the
// reference's opaque shadower path does (hit kept, minT = T_EPSILON).
void GpuDynBVH::intersect(const RenderContext& context, RayPacket& rays) const {
  const bool any = rays.getFlag(RayPacket::AnyHit);
  const int MS = RayPacket::MaxSize;
  int map[MS];
  float org[3 * MS], dir[3 * MS], tmax[MS], t[MS], u[MS], v[MS];
  int prim[MS];
  const int n = selectRays(rays, any, map);
  if (n == 0) return;
  packRays(rays, map, n, n, 0, org, dir, tmax);
  traceRays(n, org, dir, tmax, any, t, prim, u, v);
  applyHits(context, rays, any, map, n, t, prim, u, v);
}
