// GpuMeshPrimitive: see GpuMeshPrimitive.h.
#include "GpuMeshPrimitive.h"

#include <Core/Geometry/BBox.h>
#include <Interface/Context.h>
#include <Interface/RayPacket.h>

#include "GpuDynBVH.h"

using namespace Manta;

GpuMeshPrimitive::GpuMeshPrimitive(GpuDynBVH* bvh_) : accel(bvh_) {}

GpuMeshPrimitive::~GpuMeshPrimitive() {}

void GpuMeshPrimitive::preprocess(const PreprocessContext& context) { accel->preprocess(context); }

void GpuMeshPrimitive::computeBounds(const PreprocessContext& context, BBox& bbox) const {
  accel->computeBounds(context, bbox);
}

void GpuMeshPrimitive::intersect(const RenderContext& context, RayPacket& rays) const {
  accel->intersect(context, rays);
}

// Hits carry the MeshTriangle they hit; runs of rays that hit the same
// primitive get that primitive's normals (the grouping the reference's
// shading does per hit primitive).
void GpuMeshPrimitive::computeNormal(const RenderContext& context, RayPacket& rays) const {
  int i = rays.begin();
  while (i < rays.end()) {
    const Primitive* p = rays.getHitPrimitive(i);
    int e = i + 1;
    while (e < rays.end() && rays.getHitPrimitive(e) == p) ++e;
    if (p && p != this) {
      RayPacket sub(rays, i, e);
      p->computeNormal(context, sub);
    }
    i = e;
  }
}

// Texture coordinates come from the triangles' own mappers.
void GpuMeshPrimitive::setTexCoordMapper(const TexCoordMapper*) {}
