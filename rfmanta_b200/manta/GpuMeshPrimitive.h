// GpuMeshPrimitive: the Manta Primitive surface (Interface/Primitive.h:18)
// over a GpuDynBVH, so a GPU-traced triangle mesh can sit in a reference
// Group next to other objects: Group::intersect (Model/Groups/Group.cc)
// hands it each packet like any primitive.  Hits report the mesh's own
// MeshTriangle as the hit primitive (as DynBVH does), so normals, texture
// coordinates and materials come from the triangles; computeNormal here
// forwards runs of rays to the primitive each ray hit.
//
// C++98, like the rest of Manta.
#ifndef RFMANTA_B200_MANTA_GPUMESHPRIMITIVE_H
#define RFMANTA_B200_MANTA_GPUMESHPRIMITIVE_H

#include <Interface/Primitive.h>

namespace Manta {
class GpuDynBVH;

class GpuMeshPrimitive : public Primitive {
 public:
  explicit GpuMeshPrimitive(GpuDynBVH* bvh);
  virtual ~GpuMeshPrimitive();

  virtual void preprocess(const PreprocessContext& context);
  virtual void computeBounds(const PreprocessContext& context, BBox& bbox) const;
  virtual void intersect(const RenderContext& context, RayPacket& rays) const;
  virtual void computeNormal(const RenderContext& context, RayPacket& rays) const;
  virtual void setTexCoordMapper(const TexCoordMapper* new_tex);

  GpuDynBVH* bvh() const { return accel; }

 private:
  GpuDynBVH* accel;
};

}  // namespace Manta

#endif
