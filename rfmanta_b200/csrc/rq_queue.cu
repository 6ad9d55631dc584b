// rq_queue_*: one submission queue per scene for many host threads that
// each trace one small packet at a time and wait for it - the way Manta's
// render workers call DynBVH::intersect with 64-ray packets from every
// thread at once (Engine/Control/RTRT.cc:984-990, Engine/Renderers/
// Raytracer.cc:53, Engine/Shadows/HardShadows.cc:352).
//
// A per-call round trip (copy in, launch, copy out, synchronise) for 64
// rays leaves the GPU idle and the driver busy.  Here packets are gathered
// into batches instead.  A packet that finds the device idle goes out at
// once; packets that arrive while a batch is on the device fill the next
// batch, which goes out - one strided copy in, one launch, one strided copy
// out - as soon as the earlier batch has finished.  The batch size thus
// follows the load: one packet when a single thread calls, as many as are
// waiting when many do.  Each caller blocks only until its own batch is
// back, then copies its rays' results out.  Closest-hit and any-hit packets
// form separate batches (separate kernels).
//
// Per query kind there is a ring of kRing batches (at most kMaxInflight of
// them on the device at once), each with pinned host
// buffers mapped into the device's address space, laid out as rows of `cap`
// elements (org x/y/z, dir x/y/z, tmax in; t, prim, u, v out), read and
// written by the kernel directly, and its own stream and event.  States:
// FREE -> FILLING (packets copied in under the lock) -> INFLIGHT ->
// DRAINING (results back, callers copying out) -> FREE when the last caller
// is done.  A filling batch goes out as soon as fewer than kMaxInflight
// batches are on the device; the first waiter of an in-flight batch waits
// on its event outside the lock and then sends the next batch.  Each
// batch has its own condition variable, so a completion wakes only that
// batch's callers.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/rfmanta_b200.h"
#include "rq_scene.h"

namespace rq {

namespace {

constexpr int kRing = 4;
constexpr int kMaxInflight = 2;
enum QState { kFree, kFilling, kInflight, kDraining };

struct QBatch {
  float* h_in = nullptr;   // mapped pinned, 7 rows of cap
  float* h_out = nullptr;  // mapped pinned, 4 rows of cap
  float* d_in = nullptr;   // their device addresses
  float* d_out = nullptr;
  int* d_counter = nullptr;
  std::condition_variable cv;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  int count = 0;
  int users = 0;
  int state = kFree;
  bool waiting = false;  // a caller waits on `done` outside the lock
  int rc = RQ_OK;
  long long gen = 0;
};

struct QKind {
  QBatch ring[kRing];
  int filling = -1;
  int inflight = 0;  // batches on the device
};

int qfail(int code, const std::string& m) {
  set_error(m);
  return code;
}

}  // namespace

}  // namespace rq

struct rq_queue {
  rq::Scene* scene = nullptr;
  int cap = 0;
  std::mutex mu;
  std::condition_variable cv;
  rq::QKind kinds[2];
  long long batches = 0, packets = 0, rays = 0;

  ~rq_queue() {
    cudaSetDevice(scene->device);
    for (auto& k : kinds)
      for (auto& b : k.ring) {
        if (b.stream) cudaStreamSynchronize(b.stream);
        cudaFreeHost(b.h_in);
        cudaFreeHost(b.h_out);
        cudaFree(b.d_counter);
        if (b.done) cudaEventDestroy(b.done);
        if (b.stream) cudaStreamDestroy(b.stream);
      }
  }

  // Sends the filling batch of kind `any` (lock held).
  void dispatch(int any) {
    rq::QKind& K = kinds[any];
    rq::QBatch& b = K.ring[K.filling];
    b.state = rq::kInflight;
    ++K.inflight;
    K.filling = -1;
    ++batches;
    float* o = b.d_out;
    int rc = scene->trace_device(b.count, b.d_in, b.d_in + 3 * (size_t)cap,
                                 b.d_in + 6 * (size_t)cap, any != 0, o,
                                 reinterpret_cast<int32_t*>(o + cap), o + 2 * (size_t)cap,
                                 o + 3 * (size_t)cap, b.stream, b.d_counter, cap,
                                 b.count <= rq::kZeroCopyRays);
    if (rc == RQ_OK && cudaEventRecord(b.done, b.stream) != cudaSuccess) rc = RQ_ERR_CUDA;
    b.rc = rc;
    if (rc != RQ_OK) {  // nothing to wait for: the callers see the error
      b.state = rq::kDraining;
      --K.inflight;
    }
    // the batch's callers may be asleep: one of them waits on its event;
    // callers waiting for room may now start the next batch
    b.cv.notify_all();
    cv.notify_all();
  }
};

extern "C" {

int rq_queue_create(rq_scene* scene, int max_rays, rq_queue** out) {
  using namespace rq;
  if (!out) return qfail(RQ_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!scene) return qfail(RQ_ERR_ARG, "NULL scene");
  if (max_rays < 64 || max_rays > (1 << 22)) return qfail(RQ_ERR_ARG, "max_rays in [64, 4Mi]");
  if (cudaSetDevice(scene->device) != cudaSuccess) return qfail(RQ_ERR_CUDA, "cudaSetDevice");
  std::unique_ptr<rq_queue> q(new rq_queue());
  q->scene = scene;
  q->cap = max_rays;
  const size_t C = (size_t)max_rays * sizeof(float);
  for (auto& k : q->kinds)
    for (auto& b : k.ring) {
      if (cudaHostAlloc(&b.h_in, 7 * C, cudaHostAllocMapped) != cudaSuccess ||
          cudaHostAlloc(&b.h_out, 4 * C, cudaHostAllocMapped) != cudaSuccess ||
          cudaHostGetDevicePointer((void**)&b.d_in, b.h_in, 0) != cudaSuccess ||
          cudaHostGetDevicePointer((void**)&b.d_out, b.h_out, 0) != cudaSuccess ||
          cudaMalloc(&b.d_counter, sizeof(int)) != cudaSuccess ||
          cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming) != cudaSuccess)
        return qfail(RQ_ERR_OOM, "queue buffers");
    }
  *out = q.release();
  return RQ_OK;
}

int rq_queue_trace(rq_queue* q, int n, const float* org, const float* dir, const float* tmax,
                   int flags, float* t, int32_t* prim, float* u, float* v) {
  using namespace rq;
  if (!q) return qfail(RQ_ERR_ARG, "NULL queue");
  if (n < 0 || (n > 0 && (!org || !dir || !tmax))) return qfail(RQ_ERR_ARG, "bad ray arrays");
  if (flags != RQ_CLOSEST && flags != RQ_ANYHIT) return qfail(RQ_ERR_ARG, "bad flags");
  if (n == 0) return RQ_OK;
  if (n > q->cap)
    return rq_trace(static_cast<rq_scene*>(q->scene), n, org, dir, tmax, flags, t, prim, u, v);
  if (!q->scene->has_tree) return qfail(RQ_ERR_STATE, "scene has no tree");
  if (cudaSetDevice(q->scene->device) != cudaSuccess) return qfail(RQ_ERR_CUDA, "cudaSetDevice");
  const int any = flags == RQ_ANYHIT ? 1 : 0;
  const size_t cap = (size_t)q->cap;
  std::unique_lock<std::mutex> lk(q->mu);
  QKind& K = q->kinds[any];
  // a filling batch with room for n rays
  for (;;) {
    if (K.filling < 0) {
      for (int i = 0; i < kRing; ++i)
        if (K.ring[i].state == kFree) {
          K.filling = i;
          K.ring[i].state = kFilling;
          K.ring[i].count = 0;
          K.ring[i].users = 0;
          break;
        }
    }
    if (K.filling >= 0 && K.ring[K.filling].count + n <= q->cap) break;
    if (K.filling >= 0 && K.inflight < kMaxInflight) {  // full, and room on the device
      q->dispatch(any);
      continue;
    }
    q->cv.wait(lk);
  }
  const int bi = K.filling;
  QBatch& b = K.ring[bi];
  const int off = b.count;
  b.count += n;
  ++b.users;
  ++q->packets;
  q->rays += n;
  float* h = b.h_in;
  for (int c = 0; c < 3; ++c) {
    std::memcpy(h + c * cap + off, org + (size_t)c * n, n * sizeof(float));
    std::memcpy(h + (3 + c) * cap + off, dir + (size_t)c * n, n * sizeof(float));
  }
  std::memcpy(h + 6 * cap + off, tmax, n * sizeof(float));
  if (K.inflight < kMaxInflight) q->dispatch(any);  // room on the device: send now
  // wait until this batch's results are back
  for (;;) {
    if (b.state == kDraining) break;
    if (b.state == kInflight && !b.waiting) {
      b.waiting = true;
      lk.unlock();
      const cudaError_t e = cudaEventSynchronize(b.done);
      lk.lock();
      b.waiting = false;
      if (e != cudaSuccess) b.rc = RQ_ERR_CUDA;
      b.state = kDraining;
      --K.inflight;
      // the next batch goes out as soon as this one is back
      if (K.filling >= 0 && K.ring[K.filling].count > 0) q->dispatch(any);
      b.cv.notify_all();
      break;
    }
    b.cv.wait(lk);
  }
  const int rc = b.rc;
  lk.unlock();
  if (rc == RQ_OK) {
    const float* o = b.h_out;
    if (t) std::memcpy(t, o + off, n * sizeof(float));
    if (prim) std::memcpy(prim, o + cap + off, n * sizeof(int32_t));
    if (u) std::memcpy(u, o + 2 * cap + off, n * sizeof(float));
    if (v) std::memcpy(v, o + 3 * cap + off, n * sizeof(float));
  }
  lk.lock();
  if (--b.users == 0) {
    b.state = kFree;
    ++b.gen;
    q->cv.notify_all();
  }
  lk.unlock();
  if (rc != RQ_OK) return qfail(rc, "queued trace failed on the device");
  return RQ_OK;
}

int rq_queue_stats(const rq_queue* q, long long* batches, long long* packets, long long* rays) {
  if (!q) return rq::qfail(RQ_ERR_ARG, "NULL queue");
  std::lock_guard<std::mutex> g(const_cast<rq_queue*>(q)->mu);
  if (batches) *batches = q->batches;
  if (packets) *packets = q->packets;
  if (rays) *rays = q->rays;
  return RQ_OK;
}

int rq_queue_destroy(rq_queue* q) {
  delete q;
  return RQ_OK;
}

}  // extern "C"
