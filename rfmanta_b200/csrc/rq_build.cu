// GPU binned-SAH tree builder (rq_scene_build).
#include <cuda_runtime.h>

#include "../../include/rfmanta_b200.h"
#include "rq_internal.h"
#include "rq_scene.h"

extern "C" int rq_scene_build(rq_scene* scene, int bins) {
  (void)scene;
  (void)bins;
  rq::set_error("rq_scene_build: builder not available in this build");
  return RQ_ERR_STATE;
}
