// GpuHardShadows: a Manta ShadowAlgorithm (Interface/ShadowAlgorithm.h) that
// computes HardShadows' shadow rays (Engine/Shadows/HardShadows.cc:46-450)
// and traces the shadow rays of ALL lights of a packet in one GPU
// submission, through the GpuDynBVH that is the scene's object.
//
// HardShadows traces one light per call: each computeShadows call fills the
// caller's shadow packet for the next light that has a front-facing ray and
// intersects it, and the material (e.g. Lambertian::shade) calls again until
// the StateBuffer says Finished.  Here the first call (state Start) already
// computes every light's shadow packet in the reference's order (so lights
// that draw random numbers draw them in the same sequence), traces their
// rays together, and keeps the finished packets; later calls (Continuing)
// hand out the next light's packet.  The caller sees the same packets, the
// same call sequence and the same hits as with HardShadows over GpuDynBVH.
//
// Covers HardShadows with attenuateShadows off (its default, any-hit
// occlusion).  Scenes with more than kMaxLights lights are handed to
// HardShadows light by light.  The scalar (MANTA_SSE off) front-face cull
// is used; the SSE build's alignment of the first ray only widens the
// packet by masked rays.
//
// C++98, like the rest of Manta.
#ifndef RFMANTA_B200_MANTA_GPUHARDSHADOWS_H
#define RFMANTA_B200_MANTA_GPUHARDSHADOWS_H

#include <Engine/Shadows/HardShadows.h>
#include <Interface/ShadowAlgorithm.h>

#include <string>

namespace Manta {
class GpuDynBVH;

class GpuHardShadows : public ShadowAlgorithm {
 public:
  enum { kMaxLights = 16 };
  explicit GpuHardShadows(const GpuDynBVH* bvh);
  virtual ~GpuHardShadows();

  virtual void computeShadows(const RenderContext& context, StateBuffer& stateBuffer,
                              const LightSet* lights, RayPacket& source, RayPacket& shadowRays);
  virtual std::string getName() const;
  virtual std::string getSpecs() const;

 private:
  const GpuDynBVH* bvh;
  HardShadows fallback;
};

}  // namespace Manta

#endif
