// GpuDynBVH: a Manta AccelerationStructure (Interface/AccelerationStructure.h)
// whose build and ray queries run on a B200 through the rfmanta_b200 C ABI.
// Drop-in for DynBVH (Model/Groups/DynBVH.h) over a triangle Mesh.
//
// C++98, like the rest of Manta.  Link with -lrfmanta_b200.
#ifndef RFMANTA_B200_MANTA_GPUDYNBVH_H
#define RFMANTA_B200_MANTA_GPUDYNBVH_H

#include <Interface/AccelerationStructure.h>
#include <Interface/RayPacket.h>

#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"

namespace Manta {
class Group;
class Mesh;
class TexCoordMapper;

class GpuDynBVH : public AccelerationStructure {
 public:
  explicit GpuDynBVH(int device = 0, int tri_kind = RQ_TRI_WALD);
  virtual ~GpuDynBVH();

  // AccelerationStructure
  virtual void setGroup(Group* new_group);
  virtual void groupDirty();
  virtual Group* getGroup() const;
  virtual void rebuild(int proc = 0, int numProcs = 1);
  virtual void update(int proc = 0, int numProcs = 1);
  virtual void addToUpdateGraph(ObjectUpdateGraph* graph, ObjectUpdateGraphNode* parent);
  virtual bool buildFromFile(const std::string& file);
  virtual bool saveToFile(const std::string& file);

  // Object
  virtual void preprocess(const PreprocessContext& context);
  virtual void computeBounds(const PreprocessContext& context, BBox& bbox) const;
  virtual void intersect(const RenderContext& context, RayPacket& rays) const;

  // Interpolable (as DynBVH: forwarded to the group)
  virtual InterpErr parallelInterpolate(const std::vector<keyframe_t>& keyframes, int proc,
                                        int numProc);

  rq_scene* handle() const { return scene; }

  // How a packet reaches the device (setPacketMode):
  //   PerCall   every call is its own round trip (rq_trace: one launch on a
  //             private stream, rays read from and hits written to mapped
  //             host memory, one synchronise);
  //   Queue     calls go through one submission queue (rq_queue_*), where
  //             packets that arrive while the device is busy are sent
  //             together as one batch;
  //   Resident  (the default) calls go through a resident packet channel
  //             (rq_channel_*): a persistent kernel polls mapped host
  //             memory, so a packet costs no launch and no synchronise; the
  //             kernel exits 20 ms after the last packet, and while it runs
  //             device-wide synchronisation in the process waits for it.
  // setBatching(true) is Queue, setBatching(false) PerCall.  Measured under
  // Manta's Raytracer on a 16-core host, Resident is the fastest mode
  // (about 1.6x PerCall with 16 workers, 4x with 128).
  enum PacketMode { PerCall = 0, Queue = 1, Resident = 2 };
  void setPacketMode(int mode);
  void setBatching(bool on);

  // Packet plumbing shared with GpuHardShadows.  selectRays lists the rays
  // of `rays` the reference's DynBVH::intersect would trace (unmasked and,
  // for AnyHit, not yet hit) into map[] and returns their count;
  // packRays writes them as SoA rows (x, y, z of origin and direction, then
  // minT) of length `stride` at column `base`; traceRays traces such rows;
  // applyHits hands the hits back through RayPacket::hit with the real
  // MeshTriangle, its material and the scratchpad pair, and for AnyHit
  // applies the material's attenuateShadows as DynBVH does.
  int selectRays(const RayPacket& rays, bool any, int* map) const;
  static void packRays(const RayPacket& rays, const int* map, int n, int stride, int base,
                       float* org, float* dir, float* tmax);
  void traceRays(int n, const float* org, const float* dir, const float* tmax, bool any,
                 float* t, int* prim, float* u, float* v) const;
  void applyHits(const RenderContext& context, RayPacket& rays, bool any, const int* map,
                 int n, const float* t, const int* prim, const float* u, const float* v) const;

 private:
  void upload();
  void check(int rc, const char* what) const;

  Group* group;
  Mesh* mesh;
  rq_scene* scene;
  rq_queue* queue;
  rq_channel* channel;
  // each triangle's TexCoordMapper side (a cross-cast resolved once per
  // upload instead of once per hit)
  std::vector<const TexCoordMapper*> texmap;
  int device;
  int tri_kind;
  bool dirty;
  int mode;
};

}  // namespace Manta

#endif
