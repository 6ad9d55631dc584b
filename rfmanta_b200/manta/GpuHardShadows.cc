// GpuHardShadows: see GpuHardShadows.h.
#include "GpuHardShadows.h"

#include <Interface/Context.h>
#include <Interface/Light.h>
#include <Interface/LightSet.h>
#include <Interface/RayPacket.h>

#include <pthread.h>

#include <cstring>
#include <vector>

#include "GpuDynBVH.h"

using namespace Manta;

namespace {

// The finished shadow packets of one computeShadows sequence (one shade
// call), one per light: the packet data and the RayPacket fields the
// caller's packet takes over, and whether the light had a front-facing ray
// (the reference's `last != -1`).
struct ShadowSet {
  int nlights;
  RayPacketData data[GpuHardShadows::kMaxLights];
  RayPacket::PacketShape shape[GpuHardShadows::kMaxLights];
  int begin[GpuHardShadows::kMaxLights], end[GpuHardShadows::kMaxLights];
  int depth[GpuHardShadows::kMaxLights], flags[GpuHardShadows::kMaxLights];
  bool valid[GpuHardShadows::kMaxLights];
  // the one submission's rows (origin, direction, minT in; t, u, v out) and
  // hit ids, kept with the set so a shade call allocates nothing
  float rows[11 * GpuHardShadows::kMaxLights * RayPacket::MaxSize];
  int prim[GpuHardShadows::kMaxLights * RayPacket::MaxSize];
};

// Per-thread free list of ShadowSets (a shade call on a worker takes one
// at Start and returns it at Finished; nested shading takes another).
pthread_key_t g_key;
pthread_once_t g_once = PTHREAD_ONCE_INIT;

void free_list_destroy(void* p) {
  std::vector<ShadowSet*>* v = static_cast<std::vector<ShadowSet*>*>(p);
  for (size_t i = 0; i < v->size(); ++i) delete (*v)[i];
  delete v;
}

void make_key() { pthread_key_create(&g_key, free_list_destroy); }

std::vector<ShadowSet*>* free_list() {
  pthread_once(&g_once, make_key);
  std::vector<ShadowSet*>* v = static_cast<std::vector<ShadowSet*>*>(pthread_getspecific(g_key));
  if (!v) {
    v = new std::vector<ShadowSet*>();
    pthread_setspecific(g_key, v);
  }
  return v;
}

ShadowSet* take_set() {
  std::vector<ShadowSet*>* v = free_list();
  if (v->empty()) return new ShadowSet();
  ShadowSet* s = v->back();
  v->pop_back();
  return s;
}

void give_set(ShadowSet* s) { free_list()->push_back(s); }

// One light's shadow packet as HardShadows builds it (HardShadows.cc:
// 79-80 and the scalar branch 303-334): computeLight, then per ray the
// front-face test against the face-forward geometric normal; front-facing
// rays start at the hit position with no material, the others are masked
// (after the first valid ray, with that ray's origin/direction/time and
// minT 0).  Returns whether a valid ray exists; resizes to [first, last].
bool build_light_packet(const RenderContext& context, const LightSet* lights, int j,
                        RayPacket& source, RayPacket& shadowRays) {
  lights->getLight(j)->computeLight(shadowRays, context, source);
  int first = -1, last = -1;
  for (int i = source.begin(); i < source.end(); i++) {
    Vector dir = shadowRays.getDirection(i);
    if (Dot(dir, source.getFFGeometricNormal(i)) > 0) {
      shadowRays.setOrigin(i, source.getHitPosition(i));
      shadowRays.setTime(i, source.getTime(i));
      shadowRays.setHitMaterial(i, NULL);
      last = i;
      if (first < 0) first = i;
    } else if (first >= 0) {
      shadowRays.setOrigin(i, shadowRays.getOrigin(first));
      shadowRays.setDirection(i, shadowRays.getDirection(first));
      shadowRays.setTime(i, shadowRays.getTime(first));
      shadowRays.maskRay(i);
      shadowRays.overrideMinT(i, 0);
    } else {
      shadowRays.maskRay(i);
    }
  }
  if (last == -1) return false;
  shadowRays.resize(first, last + 1);
  return true;
}

}  // namespace

GpuHardShadows::GpuHardShadows(const GpuDynBVH* bvh_) : bvh(bvh_), fallback(false) {}

GpuHardShadows::~GpuHardShadows() {}

std::string GpuHardShadows::getName() const { return "gpuhard"; }

std::string GpuHardShadows::getSpecs() const { return "none"; }

void GpuHardShadows::computeShadows(const RenderContext& context, StateBuffer& stateBuffer,
                                    const LightSet* lights, RayPacket& source,
                                    RayPacket& shadowRays) {
  const int nlights = lights->numLights();
  if (nlights > kMaxLights) {
    fallback.computeShadows(context, stateBuffer, lights, source, shadowRays);
    return;
  }
  source.computeHitPositions();
  source.computeFFGeometricNormals<true>(context);
  if (stateBuffer.state == StateBuffer::Finished) return;
  ShadowSet* set = 0;
  int j = 0;
  if (stateBuffer.state == StateBuffer::Start) {
    if (nlights == 0) {
      stateBuffer.state = StateBuffer::Finished;
      return;
    }
    set = take_set();
    set->nlights = nlights;
    // every light's packet, in light order, each starting from the state
    // the caller's fresh packet has
    const int MS = RayPacket::MaxSize;
    int map[kMaxLights][RayPacket::MaxSize];
    int count[kMaxLights];
    int total = 0;
    for (int l = 0; l < nlights; ++l) {
      RayPacket p(set->data[l], shadowRays.shape, shadowRays.rayBegin, shadowRays.rayEnd,
                  shadowRays.depth, shadowRays.flags);
      p.setFlag(RayPacket::AnyHit);
      set->valid[l] = build_light_packet(context, lights, l, source, p);
      count[l] = set->valid[l] ? bvh->selectRays(p, true, map[l]) : 0;
      total += count[l];
      set->shape[l] = p.shape;
      set->begin[l] = p.rayBegin;
      set->end[l] = p.rayEnd;
      set->depth[l] = p.depth;
      set->flags[l] = p.flags;
    }
    // all lights' shadow rays in one submission
    if (total > 0) {
      float* org = set->rows;
      int* prim = set->prim;
      float* dir = org + 3 * (size_t)total;
      float* tmax = dir + 3 * (size_t)total;
      float* t = tmax + total;
      float* u = t + total;
      float* v = u + total;
      int base = 0;
      for (int l = 0; l < nlights; ++l) {
        if (!count[l]) continue;
        RayPacket p(set->data[l], set->shape[l], set->begin[l], set->end[l], set->depth[l],
                    set->flags[l]);
        GpuDynBVH::packRays(p, map[l], count[l], total, base, org, dir, tmax);
        base += count[l];
      }
      bvh->traceRays(total, org, dir, tmax, true, t, prim, u, v);
      base = 0;
      for (int l = 0; l < nlights; ++l) {
        if (!count[l]) continue;
        RayPacket p(set->data[l], set->shape[l], set->begin[l], set->end[l], set->depth[l],
                    set->flags[l]);
        bvh->applyHits(context, p, true, map[l], count[l], t + base, &prim[base], u + base,
                       v + base);
        set->flags[l] = p.flags;
        base += count[l];
      }
    }
    (void)MS;
    stateBuffer.getData<ShadowSet*>() = set;
  } else {
    set = stateBuffer.getData<ShadowSet*>();
    j = stateBuffer.i1;
  }
  // HardShadows' light loop (HardShadows.cc:79-336): from light j on, the
  // first light with a front-facing ray is this call's packet
  int l;
  do {
    l = j++;
  } while (!set->valid[l] && j < nlights);
  std::memcpy(shadowRays.data, &set->data[l], sizeof(RayPacketData));
  shadowRays.shape = set->shape[l];
  shadowRays.rayBegin = set->valid[l] ? set->begin[l] : shadowRays.rayBegin;
  shadowRays.rayEnd = set->valid[l] ? set->end[l] : shadowRays.rayEnd;
  shadowRays.depth = set->depth[l];
  shadowRays.flags = set->flags[l];
  if (j == nlights) {
    stateBuffer.state = StateBuffer::Finished;
    give_set(set);
  } else {
    stateBuffer.state = StateBuffer::Continuing;
    stateBuffer.i1 = j;
  }
}
