/*
 * rfmanta_b200 - B200 (sm_100a) ray-query path for the Manta ray tracer.
 *
 * Plain C ABI: opaque handles, plain pointers and sizes, int status codes.
 * No exception and no C++ or torch type crosses it.  A Manta build binds it
 * through the C++ drop-in classes in rfmanta_b200/manta/ (GpuDynBVH as the
 * AccelerationStructure, GpuHardShadows as the ShadowAlgorithm); Python binds
 * it through ctypes (rfmanta_b200/_lib.py).
 *
 * Arithmetic is IEEE float32 in the reference's operation order, so results
 * match the reference's MANTA_SSE=OFF build.
 *
 * Ray arrays are structure-of-arrays: org = [x0..x(n-1), y0.., z0..], the
 * same for dir.  "t" is in units of the direction vector as passed in.
 *
 * Thread safety: calls on different scenes may run concurrently.  Calls on
 * one scene may run concurrently from several host threads (the reference
 * calls DynBVH::intersect from every render worker); each call then uses its
 * own staging buffers and stream.
 */
#ifndef RFMANTA_B200_H
#define RFMANTA_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RQ_API __attribute__((visibility("default")))
#else
#define RQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (every entry point returns one). */
enum {
  RQ_OK = 0,
  RQ_ERR_ARG = 1,      /* bad argument (null pointer, bad size, bad flag) */
  RQ_ERR_CUDA = 2,     /* a CUDA call failed; see rq_last_error() */
  RQ_ERR_OOM = 3,      /* device allocation failed */
  RQ_ERR_FORMAT = 4,   /* malformed tree import (bad index, cycle, ...) */
  RQ_ERR_STATE = 5,    /* scene has no acceleration structure yet */
  RQ_ERR_CAPACITY = 6, /* tree deeper than the traversal stack supports */
  RQ_ERR_TIMEOUT = 7,  /* a bounded device wait gave up */
  RQ_ERR_NODEV = 8,    /* no usable sm_100 device */
  RQ_ERR_NOTFOUND = 9  /* a file could not be opened */
};

/* Triangle intersection kernels of the reference. */
enum {
  RQ_TRI_WALD = 0, /* WaldTriangle (Model/Primitives/WaldTriangle.cc) */
  RQ_TRI_KS = 1    /* KenslerShirleyTriangle (Model/Primitives/KenslerShirleyTriangle.cc) */
};

/* Query flags. */
enum {
  RQ_CLOSEST = 0, /* closest hit: Raytracer::traceRays -> DynBVH::intersect */
  RQ_ANYHIT = 1   /* occlusion: RayPacket::AnyHit set by HardShadows.cc:79 */
};

typedef struct rq_scene rq_scene;

/* Message of the last failed call on this host thread ("" if none). */
RQ_API const char* rq_last_error(void);

/* Library build identification: "rfmanta_b200 <version> sm_100a". */
RQ_API const char* rq_version(void);

/*
 * Uploads a triangle mesh (Mesh::vertices / vertex_indices / face_material,
 * Model/Groups/Mesh.h:27-50) to device `device`.  Replaces constructing the
 * Mesh + WaldTriangle/KenslerShirleyTriangle objects and
 * DynBVH::setGroup(Group*) (Model/Groups/DynBVH.h:150).  The scene has no
 * tree until one of the rq_scene_import_* / rq_scene_build calls.
 */
RQ_API int rq_scene_create(const float* vertices, int n_vertices,
                    const uint32_t* indices, int n_tris,
                    const uint32_t* face_material, int tri_kind, int device,
                    rq_scene** out);

RQ_API int rq_scene_destroy(rq_scene* scene);

/*
 * Imports a DynBVH tree in the reference's own byte format, the stream
 * DynBVH::saveToFile writes (Model/Groups/DynBVH.cc:2479-2501):
 *   u32 n_ids, int32 object_ids[n_ids], u32 n_nodes, BVHNode nodes[n_nodes]
 * with the x86-64 32-byte BVHNode (DynBVH.h:37-52: BBox at 0, int child at
 * 24, u8 axis at 28, isLeftCheaper bit 0 of byte 29, short children at 30).
 * Replaces DynBVH::buildFromFile (DynBVH.cc:2442-2476).  Nodes not reachable
 * from the root are ignored.
 */
RQ_API int rq_scene_import_dynbvh(rq_scene* scene, const void* blob, size_t bytes);

/*
 * Same tree given field by field: bounds[6*i] = min xyz, max xyz;
 * child[i]; children[i] (leaf iff != 0); axis[i]; left_cheaper[i];
 * object_ids[n_tris].
 */
RQ_API int rq_scene_import_tree(rq_scene* scene, int n_nodes, const float* bounds,
                         const int32_t* child, const int32_t* children,
                         const uint8_t* axis, const uint8_t* left_cheaper,
                         const int32_t* object_ids);

/*
 * Builds the tree on the GPU with a binned SAH builder (`bins` bins per
 * axis, 0 = default 32).  Replaces DynBVH::rebuild (DynBVH.cc:1699-1802);
 * reaches an SAH cost (DynBVH::computeCost, DynBVH.cc:3389-3416) within a
 * few percent of the reference's exact sweep build.
 */
RQ_API int rq_scene_build(rq_scene* scene, int bins);

/*
 * DynBVH::update (Model/Groups/DynBVH.cc:1574-1581, 2012-2123): new
 * positions for the scene's vertices (same count and triangles), the
 * triangles' precomputation redone and the tree updated on the GPU.
 *   RQ_UPDATE_ROTATE  the update as the reference ships it (TREE_ROT 1,
 *                     DynBVH.h:377): boxes refitted bottom up and, at every
 *                     internal node, leaf children of more than one object
 *                     re-split by the approximate binned build and the best
 *                     of Kopta et al.'s six tree rotations applied
 *                     (rotateNode, DynBVH.cc:3051-3348).  The tree, its
 *                     per-node costs and next free node equal those of the
 *                     reference's single-threaded DynBVH::update(0, 1) from
 *                     the same tree; the costs a tree starts from are those
 *                     the reference's rebuild leaves (computeCost<true>), for
 *                     imported trees too.  Needs a tree whose leaves hold
 *                     every triangle once.
 *   RQ_UPDATE_REFIT   boxes only, the tree's topology kept (the reference
 *                     built with TREE_ROT 0).
 * Not for two-level scenes (update the inner scenes, then create the
 * two-level scene again).
 */
#define RQ_UPDATE_REFIT 0
#define RQ_UPDATE_ROTATE 1
RQ_API int rq_scene_update_vertices_ex(rq_scene* scene, const float* vertices, int n_vertices,
                                       int mode);

/* rq_scene_update_vertices_ex with the new positions in device memory
 * (3 * n_vertices floats on the scene's device), copied on `stream` (a
 * cudaStream_t, NULL = the legacy default stream); returns when the tree is
 * updated. */
RQ_API int rq_scene_update_vertices_device(rq_scene* scene, const float* d_vertices,
                                           int n_vertices, int mode, void* stream);

/* rq_scene_update_vertices_ex(..., RQ_UPDATE_REFIT). */
RQ_API int rq_scene_update_vertices(rq_scene* scene, const float* vertices, int n_vertices);

/*
 * The state the next RQ_UPDATE_ROTATE starts from (DynBVH::costs and
 * DynBVH::nextFree, DynBVH.h:105, 382): *next_free, and when `costs` is
 * not NULL the first *next_free per-node costs (capacity >= *next_free).
 * RQ_ERR_STATE before the scene's first rotating update.
 */
RQ_API int rq_scene_update_state(const rq_scene* scene, float* costs, int capacity,
                                 int* next_free);

/*
 * Mesh files.  rq_mesh_read_ply reads a PLY file (ascii or binary) the way
 * Manta::readPlyFile does (Model/Readers/PlyReader.cc:135-269): vertex
 * x/y/z as floats moved by `transform` (3x4 row-major, NULL = identity,
 * AffineTransform::multiply_point), `vertex_indices` polygons as triangle
 * fans with face material `material`, degenerate triangles removed
 * (Mesh::removeDegenerateTriangles).  The arrays then feed rq_scene_create.
 */
typedef struct rq_mesh rq_mesh;
RQ_API int rq_mesh_read_ply(const char* path, const float* transform, uint32_t material,
                            rq_mesh** out);
RQ_API int rq_mesh_info(const rq_mesh* mesh, int* n_vertices, int* n_tris);
/* Copies 3 floats per vertex, 3 indices and 1 material per triangle; any
 * output may be NULL. */
RQ_API int rq_mesh_copy(const rq_mesh* mesh, float* vertices, uint32_t* indices,
                        uint32_t* face_material);
RQ_API int rq_mesh_destroy(rq_mesh* mesh);

/*
 * rq_mesh_read_obj reads a Wavefront OBJ file (and its mtllib) the way
 * Manta::ObjGroup does over its glm reader (Model/Groups/ObjGroup.cc:176-320,
 * Model/Readers/glm/glm.cc): vertices, triangles (polygons as fans, groups
 * newest first), each face's material index into the material table, and
 * degenerate triangles removed.  The material table is ObjGroup's: entry 0
 * its default material, entry i + 1 the library's material i (entry 1 being
 * glm's "NO_ASSIGNED_MATERIAL"), each classified as ObjGroup classifies it.
 * Texture maps are not loaded (their constant colours stand).  A missing
 * file or library is RQ_ERR_NOTFOUND, malformed data RQ_ERR_FORMAT.
 */
#define RQ_MAT_LAMBERTIAN 0  /* Lambertian(Kd) */
#define RQ_MAT_PHONG 1       /* Phong(Kd, Ks, int(Ns), reflectivity) */
#define RQ_MAT_DIELECTRIC 2  /* Ni not 0 or 1 */
#define RQ_MAT_TRANSPARENT 3 /* Tf / Tr not white, or d < 1 */
#define RQ_MAT_DEFAULT 4     /* ObjGroup's default (Lambertian of the normal) */
RQ_API int rq_mesh_read_obj(const char* path, rq_mesh** out);
/* Entries in the mesh's material table (0 for PLY meshes). */
RQ_API int rq_mesh_material_count(const rq_mesh* mesh, int* n);
/* Per entry: kind, diffuse and specular rgb, Phong exponent, reflectivity,
 * refraction index, alpha, filter rgb; any output may be NULL. */
RQ_API int rq_mesh_materials(const rq_mesh* mesh, int32_t* kind, float* diffuse,
                             float* specular, int32_t* exponent, float* reflectivity,
                             float* refraction, float* alpha, float* filter);

/* SAH cost of the scene's tree, DynBVH::computeCost<>(0) with C_isec=C_trav=1. */
RQ_API int rq_scene_sah_cost(const rq_scene* scene, double* cost);

/* Counts: internal records, leaves, maximum traversal depth. */
RQ_API int rq_scene_info(const rq_scene* scene, int* n_records, int* n_leaves,
                  int* depth, size_t* device_bytes);

/*
 * Exports the tree in the saveToFile byte format (DynBVH::saveToFile).
 * With blob == NULL only *bytes is set.
 */
RQ_API int rq_scene_export_dynbvh(const rq_scene* scene, void* blob, size_t* bytes);

/*
 * Ray query over HOST arrays (copies in, traces, copies out): the per-call
 * drop-in for DynBVH::intersect(const RenderContext&, RayPacket&) const
 * (Model/Groups/DynBVH.cc:101-272).  flags = RQ_CLOSEST or RQ_ANYHIT.
 * tmax[i] is the ray's minT on entry (RayPacket::resetHit).
 * Outputs (any may be NULL): t[i] = minT on exit (closest: hit distance or
 * tmax; any-hit: occluder distance or tmax), prim[i] = triangle index or -1,
 * u[i], v[i] = the triangle's scratchpad pair (Wald lambda/mue, KS
 * uoverd/voverd).
 */
RQ_API int rq_trace(rq_scene* scene, int n, const float* org, const float* dir,
             const float* tmax, int flags, float* t, int32_t* prim, float* u,
             float* v);

/*
 * Same query over DEVICE arrays already resident in HBM, enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream); returns without
 * synchronising.
 */
RQ_API int rq_trace_device(rq_scene* scene, int n, const float* d_org,
                    const float* d_dir, const float* d_tmax, int flags,
                    float* d_t, int32_t* d_prim, float* d_u, float* d_v,
                    void* stream);

/*
 * Submission queue for many host threads that each trace one small packet
 * at a time and wait for it: Manta's render workers call
 * DynBVH::intersect with 64-ray packets from every thread at once
 * (Engine/Control/RTRT.cc:984-990).  rq_queue_trace is rq_trace (same
 * arguments, same results) and may be called from any number of threads at
 * once.  Packets that arrive while the device works on an earlier batch are
 * gathered into the next batch, sent as one copy in, one launch and one
 * copy out as soon as the earlier batch is back; a packet that finds the
 * device idle goes out at once.  Each caller blocks until its own results
 * are back.  Packets of up to max_rays rays are batched (larger ones go
 * through rq_trace); closest-hit and any-hit packets form separate batches.
 * The scene must outlive the queue, and must not be updated while queued
 * traces run; rq_queue_destroy must not overlap calls on the queue.
 * Measured under Manta's Raytracer on a 16-core host the queue is slower
 * than per-packet rq_trace calls (waking the waiting workers costs more
 * than the launches it saves); it is kept for callers with cheaper waits.
 */
typedef struct rq_queue rq_queue;
RQ_API int rq_queue_create(rq_scene* scene, int max_rays, rq_queue** out);
RQ_API int rq_queue_trace(rq_queue* queue, int n, const float* org, const float* dir,
                          const float* tmax, int flags, float* t, int32_t* prim,
                          float* u, float* v);
/* Batches sent, packets and rays traced so far. */
RQ_API int rq_queue_stats(const rq_queue* queue, long long* batches, long long* packets,
                          long long* rays);
RQ_API int rq_queue_destroy(rq_queue* queue);

/*
 * Resident packet channel: the per-packet form of rq_trace without a launch,
 * copy or stream synchronisation per call.  A persistent kernel keeps one
 * CTA per slot resident and polls the slots, which live in mapped pinned
 * host memory; a calling thread takes a free slot, writes its rays there,
 * publishes a sequence number and spins until the device posts the hits
 * back.  rq_channel_trace has rq_trace's arguments and results and may be
 * called from any number of threads at once (up to `slots` at a time are
 * served concurrently; more wait for a slot).  Packets of more than
 * `max_rays` rays go through rq_trace.  This is the round trip Manta's
 * workers make per packet in DynBVH::intersect (Model/Groups/DynBVH.cc:
 * 101-130, called from Engine/Control/RTRT.cc:984-990).
 *
 * The kernel starts on the first packet and exits after idle_ms without a
 * packet (default 20 ms) or after life_s in all (default 10 s; the next
 * packet starts it again), or when asked (rq_channel_stop, and before any
 * entry point changes the scene's tree).  While it runs it occupies `slots`
 * CTAs of 128 threads, and device-wide synchronisation in the process
 * (cudaDeviceSynchronize, cudaFree) waits until the channel goes idle.
 * Every wait is bounded: a packet not answered within timeout_s (default
 * 10 s) returns RQ_ERR_TIMEOUT and its slot is retired.  Statistics mode
 * (rq_set_stats) does not count channel packets.  The scene must not be
 * updated while channel traces run; destroy channels before their scene
 * (a destroyed scene leaves its channels returning RQ_ERR_STATE).
 * slots <= 0 = 64 (at most 1024); max_rays <= 0 = 1024 (at most 65536).
 */
typedef struct rq_channel rq_channel;
RQ_API int rq_channel_create(rq_scene* scene, int slots, int max_rays, rq_channel** out);
RQ_API int rq_channel_trace(rq_channel* channel, int n, const float* org, const float* dir,
                            const float* tmax, int flags, float* t, int32_t* prim, float* u,
                            float* v);
RQ_API int rq_channel_set_timing(rq_channel* channel, double idle_ms, double life_s,
                                 double timeout_s);
/* Packets and rays traced through the channel, kernel launches so far, and
 * per packet on average: device time from the slot's CTA seeing the packet to
 * posting its hits, and the caller's wait from publishing it to seeing the
 * hits (any pointer may be NULL). */
RQ_API int rq_channel_stats(const rq_channel* channel, long long* packets, long long* rays,
                            long long* launches, double* device_us, double* round_trip_us);
/* Stops the kernel now (it starts again on the next packet). */
RQ_API int rq_channel_stop(rq_channel* channel);
RQ_API int rq_channel_destroy(rq_channel* channel);

/* Node-record orders a traversal can read (same records, same results):
 * the builder's depth-first pre-order, breadth-first from the root, or the
 * top 16,384 records breadth-first followed by the rest depth-first.  Batch
 * plans (rq_batch_config) and the path stages (rq_launch_config) use a
 * reordered copy the scene keeps until its tree changes; the copy is made
 * on the device by the first call that needs it, which then synchronises
 * the device once. */
#define RQ_LAYOUT_DFS 0
#define RQ_LAYOUT_BFS 1
#define RQ_LAYOUT_BFS_TOP 2

/* Traversal launch parameters (persistent kernel, warp-ballot ray fetch). */
typedef struct {
  int block_threads;    /* threads per block (multiple of 32) */
  int blocks_per_sm;    /* resident blocks per SM, 0 = occupancy maximum */
  int refill_threshold; /* idle lanes in a warp before it fetches new rays */
  int persistent;       /* 0 = one thread per ray, 1 = persistent */
  int reg_stack;        /* traversal-stack entries kept in registers (0, 1, 2, 4);
                           the rest spill to shared memory.  Path stages only. */
  int node_layout;      /* order of the node records the path stages read
                           (RQ_LAYOUT_*, taken from the RQ_PATH_EXTEND
                           config for both stages).  Path stages only. */
} rq_launch_config;

/* rq_set_launch_config / rq_get_launch_config also take these flags for the
 * path tracer's two persistent stages (rq_render_path*): block_threads,
 * blocks_per_sm, refill_threshold, reg_stack and node_layout apply,
 * `persistent` is ignored. */
#define RQ_PATH_EXTEND 2
#define RQ_PATH_SHADE 3

RQ_API int rq_set_launch_config(rq_scene* scene, int flags,
                         const rq_launch_config* cfg);
RQ_API int rq_get_launch_config(const rq_scene* scene, int flags,
                         rq_launch_config* cfg);

/*
 * Ambient light and background of a frame beyond the constant forms.  The
 * frame's `ambient` colour is ConstantAmbient's colour, or EyeAmbient's
 * (Model/AmbientLights/EyeAmbient.cc:29-44: ambient x (0.5 - 0.5 d.N_ff)
 * for ray direction d and face-forward normal N_ff).  The frame's
 * `background` colour is ConstantBackground's, or LinearBackground's `cup`
 * (Model/Backgrounds/LinearBackground.cc:15-40: cup x t + cdown x (1 - t),
 * t = 0.5 (1 + d.up), `up` normalised as the constructor does).  An all-zero
 * rq_environment selects the constant forms.
 */
#define RQ_AMBIENT_CONSTANT 0
#define RQ_AMBIENT_EYE 1
#define RQ_BACKGROUND_CONSTANT 0
#define RQ_BACKGROUND_LINEAR 1
typedef struct {
  int ambient_kind;          /* RQ_AMBIENT_* */
  int background_kind;       /* RQ_BACKGROUND_* */
  float background_down[3];  /* LinearBackground cdown */
  float background_up[3];    /* LinearBackground up (any nonzero length) */
} rq_environment;

/*
 * Whitted frame (Raytracer::traceEyeRays, Engine/Renderers/Raytracer.cc:41-97,
 * with PinholeCamera -normalizeRays, Lambertian, HardShadows and point
 * lights): the frame the reference's render workers produce tile by tile,
 * here as one device wavefront.
 */
typedef struct {
  float eye[3], lookat[3], up[3]; /* PinholeCamera -eye -lookat -up */
  float hfov, vfov;               /* degrees */
  int xres, yres;
  int n_lights;                   /* point lights, 0..16 */
  const float* lights;            /* host: n_lights x (x, y, z, r, g, b) */
  float ambient[3];               /* ConstantAmbient colour */
  float background[3];            /* ConstantBackground colour */
  int n_materials;                /* Lambertian diffuse colours by material id */
  const float* material_rgb;      /* host: n_materials x (r, g, b) */
  rq_environment environment;     /* zero = constant ambient and background */
} rq_whitted_params;

/* PinholeCamera::setup basis (Model/Cameras/PinholeCamera.cc:167-198):
 * out12 = eye, lookat-eye, u, v.  Host-only, needs no device. */
RQ_API int rq_camera_basis(const float* eye, const float* lookat, const float* up,
                           float hfov, float vfov, float* out12);

/* Renders into HOST buffers: rgb (3 per pixel, row-major from y = 0), primary
 * hit distance t and triangle id prim (-1 = miss); shadow_rays = number of
 * shadow rays sent.  t, prim, shadow_rays may be NULL. */
RQ_API int rq_render_whitted(rq_scene* scene, const rq_whitted_params* params,
                             float* rgb, float* t, int32_t* prim,
                             uint64_t* shadow_rays);

/* Same into DEVICE buffers, enqueued on `stream` without synchronising.
 * d_shadow_rays (device, may be NULL) receives the shadow-ray count. */
RQ_API int rq_render_whitted_device(rq_scene* scene, const rq_whitted_params* params,
                                    float* d_rgb, float* d_t, int32_t* d_prim,
                                    uint64_t* d_shadow_rays, void* stream);

/*
 * Batched ray queries: many batches of uneven size (closest hit or any hit)
 * over several resident scenes in one persistent launch, captured in a CUDA
 * graph.  The batched form of DynBVH::intersect that Manta's render workers
 * call per 64-ray packet (RTRT.cc:984-990).  All scenes must live on one
 * device and use one triangle kind.  Ray and output arrays are device SoA
 * as for rq_trace_device; a plan keeps the pointers, so new rays are traced
 * by writing them into the same arrays and launching the plan again.
 */
typedef struct {
  int scene;            /* index into the plan's scene array */
  int n;                /* rays in this batch */
  int flags;            /* RQ_CLOSEST or RQ_ANYHIT */
  const float* d_org;   /* device, 3 * n */
  const float* d_dir;   /* device, 3 * n */
  const float* d_tmax;  /* device, n */
  float* d_t;           /* outputs (device, n each; any may be NULL) */
  int32_t* d_prim;
  float* d_u;
  float* d_v;
} rq_batch;

typedef struct {
  int block_threads;    /* 32..256, multiple of 32 */
  int blocks_per_sm;    /* 0 = occupancy maximum */
  int chunk_rays;       /* rays a warp claims per fetch (multiple of 32) */
  int refill_threshold; /* idle lanes before a warp refills, 1..32 */
  int reg_stack;        /* traversal-stack entries kept in registers: 0, 1, 2, 4 */
  int node_layout;      /* order of the node records in HBM (RQ_LAYOUT_*) */
  int smem_entries;     /* 0 = the whole traversal stack in shared memory;
                           k in 1..64 = the first k entries of each thread in
                           shared memory and deeper ones in a global-memory
                           area the plan owns, with registers held to 48 per
                           thread, so more warps fit on an SM (reg_stack 0) */
} rq_batch_config;



typedef struct rq_batch_plan rq_batch_plan;

/* cfg NULL = defaults (128 threads, 128-ray chunks, refill 8, no register
 * stack entries, depth-first records). */
RQ_API int rq_batch_plan_create(rq_scene* const* scenes, int n_scenes,
                                const rq_batch* batches, int n_batches,
                                const rq_batch_config* cfg, rq_batch_plan** out);
/* Replays the plan's graph on `stream` (a cudaStream_t; NULL = legacy). */
RQ_API int rq_batch_plan_launch(rq_batch_plan* plan, void* stream);
RQ_API int rq_batch_plan_info(const rq_batch_plan* plan, rq_batch_config* cfg,
                              int* grid, long long* total_rays);
RQ_API int rq_batch_plan_destroy(rq_batch_plan* plan);

/* Times each candidate configuration on these batches, `reps` graph
 * replays each, and returns the fastest.  candidates NULL = the built-in
 * search: block size x rays per warp chunk x refill threshold (the
 * compaction threshold of the persistent loop) with the stack in shared
 * memory and depth-first records, then register-stack entries (0, 1, 2, 4)
 * x node layout (RQ_LAYOUT_*) at the best of those, then a short shared
 * stack column with an overflow area (smem_entries 8, 12, 16), then chunk x
 * refill again at the best stack and layout. */
RQ_API int rq_batch_autotune(rq_scene* const* scenes, int n_scenes,
                             const rq_batch* batches, int n_batches,
                             const rq_batch_config* candidates, int n_candidates,
                             int reps, rq_batch_config* best, float* best_ms);

/*
 * Served path tracing with continuous batching.  A server keeps its scenes'
 * trees resident, queues submitted render requests, admits them in arrival
 * order while their output images fit `hbm_budget_bytes`, and each step
 * packs fixed pixel chunks (chunk_pixels whole pixels, all samples) of many
 * admitted requests - different scenes, resolutions, spp and depths - into
 * one wavefront of up to path_capacity paths.  At most two steps are in
 * flight.  A request's image is identical, bit for bit, whether it ran
 * alone or with others, and identical to rq_render_path with the same
 * parameters.  All scenes share one device and triangle kind.
 */
typedef struct {
  int scene;                       /* index into the server's scenes */
  float eye[3], lookat[3], up[3];  /* PinholeCamera */
  float hfov, vfov;
  int xres, yres, spp, max_depth, rr_depth;
  uint64_t seed;
  float light_anchor[3], light_v1[3], light_v2[3], light_color[3];
  float background[3];
  float ambient[3];                /* as in rq_path_params */
  int n_materials;
  const float* material_rgb;       /* host, copied on submit */
  rq_environment environment;      /* as in rq_path_params */
} rq_serve_request;

typedef struct rq_server rq_server;

RQ_API int rq_server_create(rq_scene* const* scenes, int n_scenes,
                            long long path_capacity, int chunk_pixels,
                            size_t hbm_budget_bytes, rq_server** out);
/* Queues a request (admitted by a later rq_server_step). */
RQ_API int rq_server_submit(rq_server* server, const rq_serve_request* request,
                            int* request_id);

/*
 * Ray-query requests beside the render requests: n rays of one of the
 * server's scenes (SoA host arrays as in rq_trace, copied on submit),
 * closest or any hit.  Admitted in arrival order against the same HBM
 * budget (36 bytes per ray: the rays and their results stay on the device
 * until release), then traced in chunks of at most 1Mi rays, at most 8Mi
 * rays per step, by one persistent launch of the batched traversal kernel
 * inside the step that also runs the path chunks.  rq_server_poll reports
 * them like renders; rq_server_query_result copies t and triangle id
 * (either may be NULL) - equal, bit for bit, to rq_trace on the same rays.
 */
typedef struct {
  int scene;
  int n;
  int flags;          /* RQ_CLOSEST or RQ_ANYHIT */
  const float* org;   /* host, 3n */
  const float* dir;   /* host, 3n */
  const float* tmax;  /* host, n */
} rq_serve_query;
RQ_API int rq_server_submit_query(rq_server* server, const rq_serve_query* query,
                                  int* request_id);
RQ_API int rq_server_query_result(rq_server* server, int request_id, float* t, int32_t* prim,
                                  double* latency_s, double* queue_s);
/* Admits what fits, enqueues one step; *scheduled_paths = its path count
 * plus its ray-query rays (0 when nothing was waiting).  Blocks only to
 * keep two steps in flight. */
RQ_API int rq_server_step(rq_server* server, int* scheduled_paths);
/* Ids of requests finished on the device since the last poll. */
RQ_API int rq_server_poll(rq_server* server, int* done_ids, int max_ids, int* n_done);
/* Copies a finished request's image (rgb may be NULL) and reports its
 * latency (submit to observed completion) and its admission wait. */
RQ_API int rq_server_result(rq_server* server, int request_id, float* rgb,
                            double* latency_s, double* queue_s);
/* Frees a request's image and returns its bytes to the budget. */
RQ_API int rq_server_release(rq_server* server, int request_id);
/* ray_counts[0]: extension rays of paths plus ray-query rays; [1]: shadow
 * rays. */
RQ_API int rq_server_stats(rq_server* server, uint64_t* ray_counts, long long* steps,
                           int* pending, int* active, size_t* bytes_in_use);
RQ_API int rq_server_destroy(rq_server* server);

/* Runs a timed arrival stream through the server on the calling thread (the
 * request loop a serving front end runs; the analogue of RTRT's frame loop
 * handing out WorkQueue assignments, Engine/Control/RTRT.cc:668-1028,
 * Core/Thread/WorkQueue.cc:61-69).  Request k is submitted once
 * arrival_s[k] seconds have passed since the call began (any order), the
 * engine is stepped while it has work, and finished requests are collected
 * and released.  On return latency_s[k] and queue_s[k] hold each request's
 * latency (submit to completion observed on the host) and admission wait;
 * images (NULL, or n host pointers of which any may be NULL) receive the
 * finished images; *wall_s = first submit to last completion.  Gives up with
 * RQ_ERR_TIMEOUT after timeout_s seconds. */
RQ_API int rq_server_run_stream(rq_server* server, const rq_serve_request* requests,
                                const double* arrival_s, int n, float* const* images,
                                double* latency_s, double* queue_s, double* wall_s,
                                double timeout_s);

/* Per-step records (the server's COLLECT_STATS): with profiling on, every
 * step records the requests, chunks and distinct scenes it packed, its path
 * count, its deepest request and its device time (CUDA events on the
 * server's stream).  rq_server_profile copies up to max_steps records of
 * steps that have finished and clears them. */
typedef struct {
  int requests, chunks, scenes, max_depth;
  long long paths;
  float gpu_ms;
  double t_enqueue_s;  /* host time of the enqueue, since profiling began */
} rq_server_step_record;
RQ_API int rq_server_set_profile(rq_server* server, int on);
RQ_API int rq_server_profile(rq_server* server, rq_server_step_record* records,
                             int max_steps, int* n_steps);

/*
 * rq_render_whitted_device without any device allocation.  This entry point
 * has no counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc: a process whose device memory is already handed out to another
 * allocator, or a render thread that must not make calls which can
 * synchronise the whole device.  The frame's scratch (work counters, shadow
 * counter, material table) lives in a fixed array inside the library, so the
 * call allocates nothing; the caller still passes the outputs.  Limit:
 * n_materials <= 1024 (more return RQ_ERR_CAPACITY); any resolution
 * rq_render_whitted_device takes is accepted.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress, with that device
 * current) and caches it; make that first call before any stream capture.
 * All calls on a device share the array: calls whose work overlaps on the
 * GPU race and must be ordered by the caller (one stream, or events).
 * params->material_rgb is copied into the array on `stream` each call; give
 * it in pinned host memory or device memory so the copy is asynchronous (a
 * pageable host table is accepted, but the driver stages it and the call can
 * block).  Calls on one scene take the scene's lock, like the other frame
 * entry points, so an update on another host thread never frees the tree
 * under a frame being launched.
 */
RQ_API int rq_render_whitted_device_noalloc(rq_scene* scene,
                                            const rq_whitted_params* params,
                                            float* d_rgb, float* d_t, int32_t* d_prim,
                                            uint64_t* d_shadow_rays, void* stream);

/*
 * Two-level scene: instances of inner triangle scenes under a top-level
 * DynBVH.  inst_scene[k] indexes `inner`, inst_translation holds 3 floats
 * per instance, inst_kind[k] (NULL = all RQ_INST_TRANSLATE) is
 *   RQ_INST_TRANSLATE  an InstanceT (Model/Instances/InstanceT.cc:31-90):
 *                      rays enter with o - translation and the current minT,
 *                      a closer inner hit is taken through RayPacket::hit;
 *                      like the reference, an any-hit (shadow) query does not
 *                      report occlusion found inside it (the inner
 *                      OpaqueShadower pins minT to T_EPSILON, DynBVH.cc:
 *                      331-349, which RayPacket::hit rejects);
 *   RQ_INST_NESTED     the inner DynBVH placed in the top-level group as an
 *                      object itself (translation must be 0): hits and
 *                      occlusion as for its own triangles.
 * The top-level tree is built on the GPU over the instance boxes (inner mesh
 * bounds + translation, InstanceT::computeBounds) and can be replaced with
 * rq_scene_import_tree / rq_scene_import_dynbvh (object ids = instance
 * indices).  Inner scenes are referenced and must outlive this one; all share
 * one device and triangle kind.  Queries and frames accept the result like
 * any scene; a hit reports the inner triangle id (and, through
 * rq_trace_device_ex, the instance).
 */
#define RQ_INST_TRANSLATE 0
#define RQ_INST_NESTED 1
RQ_API int rq_scene_create_instanced(rq_scene* const* inner, int n_inner,
                                     const int32_t* inst_scene,
                                     const float* inst_translation,
                                     const int32_t* inst_kind, int n_instances,
                                     rq_scene** out);

/* rq_trace_device plus the hit instance per ray (d_inst, -1 for none or a
 * flat scene). */
RQ_API int rq_trace_device_ex(rq_scene* scene, int n, const float* d_org,
                              const float* d_dir, const float* d_tmax, int flags,
                              float* d_t, int32_t* d_prim, float* d_u, float* d_v,
                              int32_t* d_inst, void* stream);

/* Supersampled Whitted frame over a flat or instanced scene: `spp`
 * stratified jittered samples per pixel (PCG32 keyed by seed and sample),
 * averaged in sample order; spp = 1 samples pixel centres and equals
 * rq_render_whitted.  Materials are Lambertian (Model/Materials/
 * Lambertian.cc) unless material_specpow[m] >= 0: then material m is a Phong
 * (Model/Materials/Phong.cc:130-540) with diffuse material_rgb[m], specular
 * material_specular[m], that exponent and reflectivity
 * material_reflectivity[m] (NULL = none): a reflective Phong hit at depth
 * d < max_depth traces the mirrored ray with importance x reflectivity when
 * that importance's luminance exceeds importance_cutoff, and adds its colour
 * x reflectivity (Raytracer::traceRays recursion; the reference's
 * RenderParameters default to max_depth 15, importance_cutoff 0.01).  Both
 * Phong arrays NULL = all Lambertian. */
typedef struct {
  rq_whitted_params whitted;
  int spp;        /* 1, 4, 16, ... */
  uint64_t seed;
  const float* material_specular;   /* 3 per material, or NULL */
  const int32_t* material_specpow;  /* 1 per material, or NULL */
  const float* material_reflectivity; /* 1 per material, or NULL */
  int max_depth;                    /* 0..32, with material_reflectivity */
  float importance_cutoff;
} rq_frame_params;

RQ_API int rq_render_frame(rq_scene* scene, const rq_frame_params* params, float* rgb,
                           uint64_t* shadow_rays);
RQ_API int rq_render_frame_device(rq_scene* scene, const rq_frame_params* params,
                                  float* d_rgb, uint64_t* d_shadow_rays, void* stream);

/*
 * Path-traced frame: KajiyaPathtracer::traceEyeRays
 * (Engine/Renderers/KajiyaPathtracer.cc:113-302) with Lambertian materials,
 * one parallelogram AreaLight sampled with HardShadows shadow rays, cosine
 * hemisphere bounces and Russian roulette, run as a device wavefront with
 * stream compaction.  Each path draws from its own PCG32 stream keyed by
 * (seed, pixel * spp + sample), so results do not depend on batching.
 */
typedef struct {
  float eye[3], lookat[3], up[3]; /* PinholeCamera */
  float hfov, vfov;
  int xres, yres;
  int spp;                        /* 1, 4, 16, ... (stratified jitter) */
  int max_depth;                  /* bounces, primary hit = depth 0 */
  int rr_depth;                   /* Russian roulette from this depth on */
  uint64_t seed;
  float light_anchor[3];          /* Parallelogram anchor, v1, v2 */
  float light_v1[3];
  float light_v2[3];
  float light_color[3];
  float background[3];
  float ambient[3];               /* ConstantAmbient, added where a path
                                     reaches max_depth (KajiyaPathtracer's
                                     do_ambient_on_maxdepth) */
  int n_materials;
  const float* material_rgb;      /* host: n_materials x (r, g, b) */
  int chunk_paths;                /* paths per wavefront pass, 0 = 4Mi */
  rq_environment environment;     /* zero = constant ambient and background;
                                     EyeAmbient at the last bounce sees the
                                     direction sampled there, as the
                                     reference's packet holds it by then */
} rq_path_params;

/* Renders into HOST rgb (3 per pixel); ray_counts[0] = camera + bounce rays
 * traced, ray_counts[1] = shadow rays traced (may be NULL). */
RQ_API int rq_render_path(rq_scene* scene, const rq_path_params* params,
                          float* rgb, uint64_t* ray_counts);

/* Same into DEVICE rgb on `stream`, counts into d_ray_counts (2 x uint64,
 * device, may be NULL); returns without synchronising. */
RQ_API int rq_render_path_device(rq_scene* scene, const rq_path_params* params,
                                 float* d_rgb, uint64_t* d_ray_counts,
                                 void* stream);

/* Parity aid: when d_prim is set, the next path-traced frames write, per
 * bounce and path, the ray (d_org / d_dir: [3][max_depth][capacity]) and the
 * triangle it hit (d_prim: [max_depth][capacity], untouched for paths that
 * already ended).  capacity_paths must cover xres*yres*spp.  NULL turns it off. */
RQ_API int rq_set_path_debug(rq_scene* scene, int32_t* d_prim, float* d_org,
                             float* d_dir, int64_t capacity_paths);

/*
 * Profiling hook (the role of DynBVH's COLLECT_STATS counters,
 * Model/Groups/DynBVH.h:314-374): when `events` (n cudaEvent_t handles
 * created by the caller, up to 16) is set, the frame paths record events[0]
 * before their first stage and events[k] after stage k: Whitted frames
 * (rq_render_whitted*) run as one stage; path-traced frames record, for their last
 * chunk, extend and shade of every bounce (events[1 + 2d], events[2 + 2d])
 * and the resolve after them.  NULL turns it off.
 */
RQ_API int rq_set_stage_events(rq_scene* scene, void* events, int n);

/*
 * Traversal statistics (DynBVH COLLECT_STATS: node traversals and
 * intersections per ray).  d_counters is a device array of 4 uint64 the
 * frame paths add to: box tests and triangle tests of primary (or bounce)
 * rays, then of shadow rays.  Batch plans created while the first scene of
 * the plan has counters set add box and triangle tests of all their rays to
 * counters[0] and [1].  The caller zeroes it.  NULL turns counting off
 * (the default; counting builds use separate kernels).
 */
RQ_API int rq_set_stats(rq_scene* scene, uint64_t* d_counters);

/* Device time in seconds of the last rq_scene_build. */
RQ_API int rq_scene_build_seconds(const rq_scene* scene, double* seconds);

#ifdef __cplusplus
}
#endif

#endif /* RFMANTA_B200_H */
