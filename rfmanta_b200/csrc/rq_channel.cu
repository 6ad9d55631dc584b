// Resident packet channel: a persistent kernel that serves small ray packets
// written by host threads into mapped pinned memory, with no launch, copy or
// stream synchronisation per packet.
//
// Manta's render workers call AccelerationStructure::intersect with one
// packet at a time and wait for it (Engine/Control/RTRT.cc:984-990,
// Model/Groups/DynBVH.cc:101-130).  A per-call launch costs a driver launch,
// a stream synchronise and their host-side locks, tens of microseconds
// under many workers.  Here each channel slot is a mailbox in mapped host
// memory served by one resident CTA:
//
//   host (slot owner)                      device (CTA of the slot)
//   write rays, n, flags                   poll the slot's first 16 bytes
//   req = seq        (seq_cst store)         (req, stop, n, flags; one
//   load state       (seq_cst)               relaxed system-scope load)
//   spin, then yield, until done == seq    req != last: acquire fence, load
//   read hits                                rays (ld.cv), trace, store hits,
//                                            CTA barrier, done = req
//                                            (system-scope release)
//
// Lifetime.  The kernel exits when the host asks (stop), after `idle_ns`
// without a packet on any slot, or after `life_ns` in all; every device wait
// is bounded by those.  Exit is a handshake, so no packet is stranded: the
// CTA that decides first marks the channel EXITING in mapped memory, issues
// a system-scope sequentially consistent fence and raises a device flag;
// each CTA then looks at its slot once more before it returns.  A host
// thread publishes its request with a sequentially consistent store and then
// reads the state: either it sees EXITING (it relaunches the kernel, after
// the old one has finished, unless the last look served it) or the last look
// sees its request.  Relaunches are serialised by a host mutex and counted
// by an epoch.
//
// A running channel kernel keeps the device busy: device-wide
// synchronisation in the process (cudaDeviceSynchronize, cudaFree) waits
// until the channel goes idle.  Entry points that change a scene's tree stop
// the scene's channels first (park_channels).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstddef>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_scene.h"
#include "rq_traverse.cuh"

namespace rq {

namespace {

constexpr int kChanThreads = 128;
constexpr int kStateIdle = 0;
constexpr int kStateRunning = 1;
constexpr int kStateExiting = 2;

// One slot's header in mapped host memory: the host-written half and the
// device-written half on separate 128-byte lines.
struct alignas(128) ChanHdr {
  unsigned req;   // sequence number of the slot's newest request (written last)
  unsigned stop;  // set by the host (on every slot) to make the kernel exit
  int n;          // rays of the request
  int flags;      // RQ_CLOSEST or RQ_ANYHIT
  int pad0[28];
  unsigned done;  // sequence number of the newest request served
  unsigned serve_ns;  // device time of that request, from seeing it to posting it
  int pad1[30];
};
static_assert(sizeof(ChanHdr) == 256, "two 128-byte halves");
static_assert(offsetof(ChanHdr, flags) == 12 && offsetof(ChanHdr, done) == 128,
              "req, stop, n, flags in the first 16 bytes; done on the second line");

struct alignas(128) ChanCtl {
  int state;  // kState*: RUNNING set by the host at launch, EXITING by the kernel
  int pad[31];
};

// Device-memory control block, cleared before every launch.
struct ChanDev {
  unsigned long long last_active;  // globaltimer of the newest packet served
  int exit_claim;                  // the CTA that decides the exit
  int exit_go;                     // raised once the state says EXITING
};

struct ChanArgs {
  DevScene S;
  ChanHdr* hdr;
  float4* data;  // slot k: data + k * 3 * max_rays (2 float4 in, 1 out per ray)
  ChanCtl* ctl;
  ChanDev* dev;
  int max_rays;
  unsigned long long idle_ns;
  unsigned long long life_ns;
};

__device__ __forceinline__ unsigned ld_acquire_sys(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// req, stop, n and flags of a slot in one 16-byte load: one PCIe read of
// one cache line, which the host wrote in the order n, flags, req
__device__ __forceinline__ uint4 ld_relaxed_sys_v4(const unsigned* p) {
  uint4 v;
  asm volatile("ld.relaxed.sys.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p)
               : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_sys() {
  asm volatile("fence.acq_rel.sys;" ::: "memory");
}
__device__ __forceinline__ void st_release_sys(unsigned* p, unsigned v) {
  asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_sys(int* p, int v) {
  asm volatile("st.relaxed.sys.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_sc_sys() { asm volatile("fence.sc.sys;" ::: "memory"); }
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Traces packet rays [0, n) of one slot: per ray two float4 in `in`
// (origin, minT; direction, 0) and one float4 out (t, triangle id bits, u,
// v), so a ray costs two loads and one store across PCIe.  Rays are read
// with ld.cv (the host rewrites them for every request).
template <int KIND, bool ANY>
__device__ __forceinline__ void serve_rays(const DevScene& S, const float4* in, float4* out,
                                           int n, int2* stk) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float4 a = __ldcv(in + 2 * i);
    const float4 b = __ldcv(in + 2 * i + 1);
    Ray r;
    r.o[0] = a.x;
    r.o[1] = a.y;
    r.o[2] = a.z;
    r.minT = a.w;
    r.d[0] = b.x;
    r.d[1] = b.y;
    r.d[2] = b.z;
#pragma unroll
    for (int c = 0; c < 3; ++c) r.inv[c] = fdiv(1.f, r.d[c]);  // RayPacket.cc:106-110
    Hit h;
    int ref, sp;
    start_ray(S, r, h, ref, sp);
    while (ref != kDone) step<KIND, ANY>(S, r, h, ref, sp, stk, blockDim.x);
    out[i] = make_float4(h.t, __int_as_float(h.id), h.u, h.v);
  }
}

template <int KIND>
__global__ void __launch_bounds__(kChanThreads) channel_kernel(ChanArgs A) {
  extern __shared__ int2 stk[];
  __shared__ unsigned s_req;
  __shared__ int s_cmd, s_n, s_any;
  __shared__ unsigned long long s_t;
  ChanHdr* h = A.hdr + blockIdx.x;
  const float4* in = A.data + (size_t)blockIdx.x * 3 * A.max_rays;
  float4* out = A.data + (size_t)blockIdx.x * 3 * A.max_rays + (size_t)2 * A.max_rays;
  unsigned last = 0;
  bool sweep = false;
  unsigned long long t0 = 0;
  unsigned quiet = 0;  // empty looks at the slot since its last packet
  if (threadIdx.x == 0) {
    last = ld_acquire_sys(&h->done);
    t0 = now_ns();
  }
  for (;;) {
    if (threadIdx.x == 0) {
      int cmd = 0;  // 0 = look again, 1 = serve, 2 = exit
      // a relaxed look at the slot's own line (request and stop word); the
      // acquire fence only once a packet is there.  Each CTA reads only its
      // own slot across PCIe: lines read by every CTA at once serialise.
      const uint4 rs = ld_relaxed_sys_v4(&h->req);
      const unsigned req = rs.x;
      if (req != last) {
        fence_acq_rel_sys();
        cmd = 1;
        quiet = 0;
        s_t = now_ns();
        s_req = req;
        s_n = min(max((int)rs.z, 0), A.max_rays);
        s_any = (int)rs.w == RQ_ANYHIT;
      } else if (sweep) {
        cmd = 2;
      } else if (*(volatile int*)&A.dev->exit_go) {
        // the channel is EXITING: one more look at the slot, then return
        fence_sc_sys();
        sweep = true;
      } else {
        // (another CTA may have stamped last_active after this CTA read
        // the timer: compare before subtracting)
        const unsigned long long now = now_ns();
        const unsigned long long la =
            max(t0, *(volatile unsigned long long*)&A.dev->last_active);
        const bool idle = now > la && now - la > A.idle_ns;
        const bool old = now > t0 && now - t0 > A.life_ns;
        if (rs.y != 0u || idle || old) {
          if (atomicCAS(&A.dev->exit_claim, 0, 1) == 0) {
            st_relaxed_sys(&A.ctl->state, kStateExiting);
            fence_sc_sys();
            atomicExch(&A.dev->exit_go, 1);
          }
        } else {
          // a slot in use is looked at about every microsecond (one PCIe
          // read); one left alone backs off to ~8 us, so unused slots do not
          // crowd the link
          ++quiet;
          __nanosleep(quiet < 512 ? 32 : (quiet < 4096 ? 1024 : 8192));
        }
      }
      s_cmd = cmd;
    }
    __syncthreads();
    const int cmd = s_cmd;
    if (cmd == 2) break;
    if (cmd == 1) {
      int2* col = stk + threadIdx.x;
      if (s_any) serve_rays<KIND, true>(A.S, in, out, s_n, col);
      else serve_rays<KIND, false>(A.S, in, out, s_n, col);
      // the CTA's hit stores are ordered before thread 0's release of
      // `done` by the barrier; the release at system scope is cumulative
      __syncthreads();
      if (threadIdx.x == 0) {
        h->serve_ns = (unsigned)min(now_ns() - s_t, 0xffffffffull);
        st_release_sys(&h->done, s_req);
        last = s_req;
        atomicMax(&A.dev->last_active, now_ns());
      }
    }
    __syncthreads();
  }
}

inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#endif
}

}  // namespace
}  // namespace rq

struct rq_channel {
  std::atomic<rq::Scene*> scene{nullptr};  // NULL once the scene is gone
  int device = 0;
  int slots = 0;
  int max_rays = 0;
  unsigned long long idle_ns = 0;
  unsigned long long life_ns = 0;
  double timeout_s = 10.0;
  // mapped pinned host memory
  rq::ChanHdr* hdr = nullptr;
  rq::ChanCtl* ctl = nullptr;
  float4* data = nullptr;
  rq::ChanDev* d_dev = nullptr;
  cudaStream_t stream = nullptr;
  std::atomic<int> retired{0};               // slots given up after a timeout (kept busy)
  // launches
  std::mutex launch_mu;
  std::atomic<unsigned> epoch{0};
  bool launched = false;
  uint64_t launched_gen = ~0ull;
  std::atomic<long long> launches{0};
  // host-side state of each slot on its own cache line, so callers on
  // different slots share no line: the owner flag, the last request's
  // sequence number and counters written only by the slot's current owner
  // (summed when read)
  struct alignas(64) Slot {
    std::atomic<int> busy{0};
    unsigned seq = 0;
    std::atomic<long long> packets{0}, rays{0}, device_ns{0}, wait_ns{0};
  };
  std::unique_ptr<Slot[]> slot;

  ~rq_channel();
};

namespace rq {
namespace {

int cfail(int code, const std::string& m) {
  set_error(m);
  return code;
}

int state_of(const rq_channel* ch) { return __atomic_load_n(&ch->ctl->state, __ATOMIC_SEQ_CST); }

// Stops the running kernel, if any, and waits for it (launch_mu held).
int stop_locked(rq_channel* ch) {
  if (!ch->launched) return RQ_OK;
  for (int k = 0; k < ch->slots; ++k) __atomic_store_n(&ch->hdr[k].stop, 1u, __ATOMIC_SEQ_CST);
  cudaSetDevice(ch->device);
  const cudaError_t e = cudaStreamSynchronize(ch->stream);
  ch->launched = false;
  __atomic_store_n(&ch->ctl->state, kStateIdle, __ATOMIC_SEQ_CST);
  if (e != cudaSuccess) return cfail(RQ_ERR_CUDA, std::string("channel: ") + cudaGetErrorString(e));
  return RQ_OK;
}

// Launches the kernel unless another thread did since `seen_epoch` was
// read; waits for an exiting kernel first.
int relaunch(rq_channel* ch, unsigned seen_epoch) {
  std::lock_guard<std::mutex> g(ch->launch_mu);
  if (ch->epoch.load(std::memory_order_acquire) != seen_epoch) return RQ_OK;
  if (!ch->scene.load()) return cfail(RQ_ERR_STATE, "channel: its scene was destroyed");
  if (cudaSetDevice(ch->device) != cudaSuccess) return cfail(RQ_ERR_CUDA, "cudaSetDevice");
  if (ch->launched) {
    const cudaError_t e = cudaStreamSynchronize(ch->stream);
    ch->launched = false;
    if (e != cudaSuccess)
      return cfail(RQ_ERR_CUDA, std::string("channel: ") + cudaGetErrorString(e));
  }
  Scene* s = ch->scene.load();
  if (!s->has_tree) return cfail(RQ_ERR_STATE, "scene has no tree");
  ChanArgs A;
  A.S = s->dev();
  A.hdr = ch->hdr;
  A.data = ch->data;
  A.ctl = ch->ctl;
  A.dev = ch->d_dev;
  A.max_rays = ch->max_rays;
  A.idle_ns = ch->idle_ns;
  A.life_ns = ch->life_ns;
  const size_t smem = (size_t)std::max(1, A.S.depth) * kChanThreads * sizeof(int2);
  const void* f = s->tri_kind == kWald ? (const void*)channel_kernel<kWald>
                                       : (const void*)channel_kernel<kKS>;
  if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return cfail(RQ_ERR_CAPACITY, "channel: traversal stack does not fit in shared memory");
  cudaError_t e = cudaMemsetAsync(ch->d_dev, 0, sizeof(ChanDev), ch->stream);
  if (e != cudaSuccess) return cfail(RQ_ERR_CUDA, std::string("channel: ") + cudaGetErrorString(e));
  for (int k = 0; k < ch->slots; ++k) __atomic_store_n(&ch->hdr[k].stop, 0u, __ATOMIC_SEQ_CST);
  __atomic_store_n(&ch->ctl->state, kStateRunning, __ATOMIC_SEQ_CST);
  if (s->tri_kind == kWald)
    channel_kernel<kWald><<<ch->slots, kChanThreads, smem, ch->stream>>>(A);
  else
    channel_kernel<kKS><<<ch->slots, kChanThreads, smem, ch->stream>>>(A);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    __atomic_store_n(&ch->ctl->state, kStateIdle, __ATOMIC_SEQ_CST);
    return cfail(RQ_ERR_CUDA, std::string("channel launch: ") + cudaGetErrorString(e));
  }
  ch->launched = true;
  ch->launched_gen = s->generation;
  ch->launches.fetch_add(1);
  ch->epoch.fetch_add(1, std::memory_order_release);
  return RQ_OK;
}

// A free slot for this thread (the one it used last when free); -1 when
// every slot was given up after a timeout.
int take_slot(rq_channel* ch) {
  static thread_local int hint = -1;
  const int n = ch->slots;
  int start = hint >= 0 && hint < n ? hint : (int)(std::hash<std::thread::id>()(
                                                       std::this_thread::get_id()) % n);
  for (unsigned spin = 0;; ++spin) {
    if (ch->retired.load(std::memory_order_relaxed) == n) return -1;
    for (int k = 0; k < n; ++k) {
      const int i = (start + k) % n;
      int zero = 0;
      if (ch->slot[i].busy.load(std::memory_order_relaxed) == 0 &&
          ch->slot[i].busy.compare_exchange_strong(zero, 1, std::memory_order_acquire)) {
        hint = i;
        return i;
      }
    }
    if (spin > 64) std::this_thread::yield();
    else cpu_relax();
  }
}

}  // namespace

void park_channels(Scene* s) {
  std::lock_guard<std::mutex> g(s->chan_mu);
  for (rq_channel* ch : s->channels) {
    std::lock_guard<std::mutex> l(ch->launch_mu);
    stop_locked(ch);
  }
}

void detach_channels(Scene* s) {
  std::lock_guard<std::mutex> g(s->chan_mu);
  for (rq_channel* ch : s->channels) {
    std::lock_guard<std::mutex> l(ch->launch_mu);
    stop_locked(ch);
    ch->scene.store(nullptr);
  }
  s->channels.clear();
}

}  // namespace rq

rq_channel::~rq_channel() {
  {
    std::lock_guard<std::mutex> l(launch_mu);
    if (ctl) rq::stop_locked(this);
  }
  if (rq::Scene* s = scene.load()) {
    std::lock_guard<std::mutex> g(s->chan_mu);
    auto& v = s->channels;
    v.erase(std::remove(v.begin(), v.end(), this), v.end());
  }
  cudaSetDevice(device);
  if (stream) cudaStreamDestroy(stream);
  if (d_dev) cudaFree(d_dev);
  if (hdr) cudaFreeHost(hdr);
  if (data) cudaFreeHost(data);
}

extern "C" {

int rq_channel_create(rq_scene* scene, int slots, int max_rays, rq_channel** out) {
  using namespace rq;
  if (!out) return cfail(RQ_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!scene) return cfail(RQ_ERR_ARG, "NULL scene");
  Scene* s = scene;
  if (s->instanced) return cfail(RQ_ERR_ARG, "channels take triangle scenes");
  if (slots <= 0) slots = 64;
  if (slots > 1024) return cfail(RQ_ERR_ARG, "1..1024 slots");
  if (max_rays <= 0) max_rays = 1024;
  if (max_rays > 65536) return cfail(RQ_ERR_ARG, "max_rays must be at most 65536");
  if (cudaSetDevice(s->device) != cudaSuccess) return cfail(RQ_ERR_CUDA, "cudaSetDevice");
  std::unique_ptr<rq_channel> ch(new rq_channel());
  ch->device = s->device;
  ch->slots = slots;
  ch->max_rays = max_rays;
  ch->idle_ns = 20ull * 1000 * 1000;        // 20 ms without a packet
  ch->life_ns = 10ull * 1000 * 1000 * 1000;  // 10 s per launch
  void* p = nullptr;
  const size_t hb = sizeof(ChanHdr) * slots + sizeof(ChanCtl);
  if (cudaHostAlloc(&p, hb, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
    return cfail(RQ_ERR_OOM, "channel headers");
  std::memset(p, 0, hb);
  ch->hdr = static_cast<ChanHdr*>(p);
  ch->ctl = reinterpret_cast<ChanCtl*>(ch->hdr + slots);
  const size_t db = (size_t)slots * 3 * max_rays * sizeof(float4);
  if (cudaHostAlloc(&p, db, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
    return cfail(RQ_ERR_OOM, "channel packet buffers");
  ch->data = static_cast<float4*>(p);
  // device views of the mapped buffers (the same addresses under UVA)
  void* dp = nullptr;
  if (cudaHostGetDevicePointer(&dp, ch->hdr, 0) != cudaSuccess || dp != (void*)ch->hdr ||
      cudaHostGetDevicePointer(&dp, ch->data, 0) != cudaSuccess || dp != (void*)ch->data)
    return cfail(RQ_ERR_CUDA, "channel buffers are not mapped at their host addresses");
  if (cudaMalloc(&ch->d_dev, sizeof(ChanDev)) != cudaSuccess)
    return cfail(RQ_ERR_OOM, "channel control block");
  if (cudaStreamCreateWithFlags(&ch->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cfail(RQ_ERR_CUDA, "channel stream");
  ch->slot.reset(new rq_channel::Slot[slots]);
  ch->scene.store(s);
  {
    std::lock_guard<std::mutex> g(s->chan_mu);
    s->channels.push_back(ch.get());
  }
  *out = ch.release();
  return RQ_OK;
}

int rq_channel_set_timing(rq_channel* ch, double idle_ms, double life_s, double timeout_s) {
  using namespace rq;
  if (!ch) return cfail(RQ_ERR_ARG, "NULL channel");
  if (!(idle_ms > 0) || !(life_s > 0) || !(timeout_s > 0) || life_s > 3600.0 ||
      idle_ms > 1e6)
    return cfail(RQ_ERR_ARG, "timings must be positive (life_s <= 3600)");
  std::lock_guard<std::mutex> l(ch->launch_mu);
  ch->idle_ns = (unsigned long long)(idle_ms * 1e6);
  ch->life_ns = (unsigned long long)(life_s * 1e9);
  ch->timeout_s = timeout_s;
  // a running kernel keeps the old timings until it next exits
  return RQ_OK;
}

int rq_channel_trace(rq_channel* ch, int n, const float* org, const float* dir,
                     const float* tmax, int flags, float* t, int32_t* prim, float* u, float* v) {
  using namespace rq;
  if (!ch) return cfail(RQ_ERR_ARG, "NULL channel");
  if (n < 0 || (n > 0 && (!org || !dir || !tmax))) return cfail(RQ_ERR_ARG, "bad ray arrays");
  if (flags != RQ_CLOSEST && flags != RQ_ANYHIT) return cfail(RQ_ERR_ARG, "bad flags");
  if (n == 0) return RQ_OK;
  Scene* s = ch->scene.load();
  if (!s) return cfail(RQ_ERR_STATE, "channel: its scene was destroyed");
  if (n > ch->max_rays)  // larger packets take the per-call path
    return rq_trace(static_cast<rq_scene*>(s), n, org, dir, tmax, flags, t, prim, u, v);
  if (!s->has_tree) return cfail(RQ_ERR_STATE, "scene has no tree");
  if (ch->launched && s->generation != ch->launched_gen) {
    // a new tree since the kernel started: stop it; the wait below starts
    // one with the new descriptor
    std::lock_guard<std::mutex> l(ch->launch_mu);
    if (ch->launched && s->generation != ch->launched_gen) {
      const int rc = stop_locked(ch);
      if (rc != RQ_OK) return rc;
    }
  }
  const int k = take_slot(ch);
  if (k < 0) return cfail(RQ_ERR_STATE, "channel: every slot timed out");
  ChanHdr* h = ch->hdr + k;
  // per ray: (origin, minT), (direction, 0) in; (t, id bits, u, v) out
  float4* in = ch->data + (size_t)k * 3 * ch->max_rays;
  const float4* res = in + (size_t)2 * ch->max_rays;
  for (int i = 0; i < n; ++i) {
    in[2 * i] = make_float4(org[i], org[n + i], org[2 * (size_t)n + i], tmax[i]);
    in[2 * i + 1] = make_float4(dir[i], dir[n + i], dir[2 * (size_t)n + i], 0.f);
  }
  h->n = n;
  h->flags = flags;
  h->serve_ns = 0;
  const unsigned seq = ++ch->slot[k].seq;
  const auto t0 = std::chrono::steady_clock::now();
  __atomic_store_n(&h->req, seq, __ATOMIC_SEQ_CST);
  int rc = RQ_OK;
  for (unsigned it = 1;; ++it) {
    if (__atomic_load_n(&h->done, __ATOMIC_ACQUIRE) == seq) break;
    const unsigned ep = ch->epoch.load(std::memory_order_acquire);
    if (state_of(ch) != kStateRunning) {
      rc = relaunch(ch, ep);
      if (rc != RQ_OK) break;
      continue;
    }
    // spin for the first ~1 us of the wait, then offer the core to other
    // runnable threads between looks (render workers outnumbering the cores
    // keep shading while this one waits; with no other thread ready the
    // yield returns at once)
    if (it < 16) {
      cpu_relax();
    } else {
      if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >
          ch->timeout_s) {
        rc = cfail(RQ_ERR_TIMEOUT, "channel: no answer from the device");
        break;
      }
      std::this_thread::yield();
    }
  }
  if (rc != RQ_OK) {
    // the request may still be served later: the slot stays taken for good
    ch->retired.fetch_add(1);
    return rc;
  }
  for (int i = 0; i < n; ++i) {
    const float4 r = res[i];
    if (t) t[i] = r.x;
    if (prim) std::memcpy(prim + i, &r.y, sizeof(int32_t));
    if (u) u[i] = r.z;
    if (v) v[i] = r.w;
  }
  rq_channel::Slot& ss = ch->slot[k];
  ss.device_ns.store(ss.device_ns.load(std::memory_order_relaxed) + h->serve_ns,
                     std::memory_order_relaxed);
  ss.wait_ns.store(ss.wait_ns.load(std::memory_order_relaxed) +
                       std::chrono::duration_cast<std::chrono::nanoseconds>(
                           std::chrono::steady_clock::now() - t0)
                           .count(),
                   std::memory_order_relaxed);
  ss.packets.store(ss.packets.load(std::memory_order_relaxed) + 1, std::memory_order_relaxed);
  ss.rays.store(ss.rays.load(std::memory_order_relaxed) + n, std::memory_order_relaxed);
  ss.busy.store(0, std::memory_order_release);
  return RQ_OK;
}

int rq_channel_stats(const rq_channel* ch, long long* packets, long long* rays,
                     long long* launches, double* device_us, double* round_trip_us) {
  if (!ch) return rq::cfail(RQ_ERR_ARG, "NULL channel");
  long long p = 0, r = 0, dn = 0, wn = 0;
  for (int k = 0; k < ch->slots; ++k) {
    p += ch->slot[k].packets.load(std::memory_order_relaxed);
    r += ch->slot[k].rays.load(std::memory_order_relaxed);
    dn += ch->slot[k].device_ns.load(std::memory_order_relaxed);
    wn += ch->slot[k].wait_ns.load(std::memory_order_relaxed);
  }
  if (packets) *packets = p;
  if (rays) *rays = r;
  if (launches) *launches = ch->launches.load();
  if (device_us) *device_us = p ? dn * 1e-3 / p : 0.0;
  if (round_trip_us) *round_trip_us = p ? wn * 1e-3 / p : 0.0;
  return RQ_OK;
}

int rq_channel_stop(rq_channel* ch) {
  if (!ch) return rq::cfail(RQ_ERR_ARG, "NULL channel");
  std::lock_guard<std::mutex> l(ch->launch_mu);
  return rq::stop_locked(ch);
}

int rq_channel_destroy(rq_channel* ch) {
  delete ch;
  return RQ_OK;
}

}  // extern "C"
