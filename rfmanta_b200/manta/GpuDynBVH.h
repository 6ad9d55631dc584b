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

#include "../../include/rfmanta_b200.h"

namespace Manta {
class Group;
class Mesh;

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

 private:
  void upload();
  void check(int rc, const char* what) const;

  Group* group;
  Mesh* mesh;
  rq_scene* scene;
  int device;
  int tri_kind;
  bool dirty;
};

}  // namespace Manta

#endif
