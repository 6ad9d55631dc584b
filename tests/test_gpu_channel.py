"""The resident packet channel (rq_channel_*): a persistent kernel serving
small packets that host threads write into mapped memory, the way Manta's
render workers call DynBVH::intersect one packet at a time.  Every packet's
results equal rq_trace's on the same rays, bit for bit, from many threads at
once, for closest and any hit; packets beyond the channel's size go through
rq_trace; the kernel's idle exit, lifetime exit and restarts lose no packet;
a scene update or rebuild reaches the channel; a destroyed scene leaves the
channel returning RQ_ERR_STATE."""
import ctypes as C
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _trace(fn, h, o, d, tm, flags):
    n = tm.shape[0]
    out = dict(t=np.zeros(n, np.float32), prim=np.zeros(n, np.int32),
               u=np.zeros(n, np.float32), v=np.zeros(n, np.float32))
    rc = fn(h, n, _p(o), _p(d), _p(tm), flags, _p(out["t"]), _p(out["prim"]), _p(out["u"]),
            _p(out["v"]))
    return rc, out


def _same(got, want):
    if not np.array_equal(got["prim"], want["prim"]):
        return False
    return all(np.array_equal(got[f].view(np.uint32), want[f].view(np.uint32))
               for f in ("t", "u", "v"))


def _packets(mesh, count, sizes, seed0=0):
    from rfmanta_b200 import _lib, scenes
    lo, hi = mesh.bounds()
    out = []
    for k in range(count):
        n = sizes[k % len(sizes)]
        any_ = k % 3 == 0
        o, d, tm, _ = scenes.random_rays(n, lo - 0.3, hi + 0.3, seed=seed0 + k,
                                         anyhit_fraction=1.0 if any_ else 0.0)
        if not any_:
            tm = np.full(n, 1e19, np.float32)
        out.append((np.ascontiguousarray(o), np.ascontiguousarray(d), np.ascontiguousarray(tm),
                    _lib.RQ_ANYHIT if any_ else _lib.RQ_CLOSEST))
    return out


def _run_threads(fn, ch, packets, nthreads):
    from rfmanta_b200 import _lib
    results = [None] * len(packets)
    errors = []

    def worker(w):
        for k in range(w, len(packets), nthreads):
            o, d, tm, fl = packets[k]
            rc, out = _trace(fn, ch, o, d, tm, fl)
            if rc != _lib.RQ_OK:
                errors.append((k, rc, _lib.lib.rq_last_error()))
            results[k] = out

    th = [threading.Thread(target=worker, args=(w,)) for w in range(nthreads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return results, errors


def _stats(ch):
    from rfmanta_b200 import _lib
    p, r, n = C.c_longlong(), C.c_longlong(), C.c_longlong()
    dev, rt = C.c_double(), C.c_double()
    _lib.check(_lib.lib.rq_channel_stats(ch, C.byref(p), C.byref(r), C.byref(n), C.byref(dev),
                                         C.byref(rt)))
    assert (dev.value > 0) == (p.value > 0) and rt.value >= dev.value
    return p.value, r.value, n.value


@pytest.fixture(scope="module")
def scene():
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.small_frame_scene(level=5, grid=60)
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    return sc, bvh


@pytest.mark.parametrize("kind", [0, 1])
def test_channel_matches_plain_trace_across_threads(kind):
    from rfmanta_b200 import _lib, scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.small_frame_scene(level=5, grid=60)
    bvh = GpuDynBVH(tri_kind=kind)
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    ch = C.c_void_p()
    # 8 slots for 24 threads (threads wait for slots); 256-ray packets at most
    _lib.check(_lib.lib.rq_channel_create(bvh.handle, 8, 256, C.byref(ch)))
    packets = _packets(sc.mesh, 24 * 10, [64, 1, 37, 64, 5, 129, 256])
    packets += _packets(sc.mesh, 1, [700], seed0=5000)  # beyond max_rays: rq_trace
    results, errors = _run_threads(_lib.lib.rq_channel_trace, ch, packets, 24)
    assert not errors, errors
    for k, (o, d, tm, fl) in enumerate(packets):
        rc, want = _trace(_lib.lib.rq_trace, bvh.handle, o, d, tm, fl)
        assert rc == _lib.RQ_OK
        assert _same(results[k], want), k
    p, r, n = _stats(ch)
    assert p == len(packets) - 1  # the oversized packet bypasses the channel
    assert r == sum(int(x[2].shape[0]) for x in packets[:-1])
    assert n >= 1
    _lib.check(_lib.lib.rq_channel_destroy(ch))


def test_channel_idle_exit_and_lifetime_restarts(scene):
    """A short idle limit and lifetime make the kernel exit and start again
    many times while four threads keep sending packets: none is lost and
    every result equals rq_trace's."""
    from rfmanta_b200 import _lib
    sc, bvh = scene
    ch = C.c_void_p()
    _lib.check(_lib.lib.rq_channel_create(bvh.handle, 4, 64, C.byref(ch)))
    _lib.check(_lib.lib.rq_channel_set_timing(ch, 1.0, 0.02, 10.0))
    packets = _packets(sc.mesh, 4 * 150, [64, 17, 3], seed0=100)
    stop = time.time() + 0.5
    results = [None] * len(packets)
    errors = []

    def worker(w):
        k = w
        while k < len(packets):
            o, d, tm, fl = packets[k]
            rc, out = _trace(_lib.lib.rq_channel_trace, ch, o, d, tm, fl)
            if rc != _lib.RQ_OK:
                errors.append((k, rc))
            results[k] = out
            k += 4
            if k % 40 < 4 and time.time() < stop:
                time.sleep(0.003)  # past the 1 ms idle limit

    th = [threading.Thread(target=worker, args=(w,)) for w in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for k, (o, d, tm, fl) in enumerate(packets):
        rc, want = _trace(_lib.lib.rq_trace, bvh.handle, o, d, tm, fl)
        assert _same(results[k], want), k
    _, _, launches = _stats(ch)
    assert launches >= 2
    # explicit stop, then the next packet starts the kernel again
    _lib.check(_lib.lib.rq_channel_stop(ch))
    o, d, tm, fl = packets[1]
    rc, out = _trace(_lib.lib.rq_channel_trace, ch, o, d, tm, fl)
    assert rc == _lib.RQ_OK and _same(out, _trace(_lib.lib.rq_trace, bvh.handle, o, d, tm, fl)[1])
    assert _stats(ch)[2] == launches + 1
    _lib.check(_lib.lib.rq_channel_destroy(ch))


def test_channel_follows_scene_changes():
    """Rotating updates and a rebuild stop the channel's kernel; its next
    packets trace the new tree."""
    from rfmanta_b200 import _lib, scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.small_frame_scene(level=3, grid=10)
    mesh = sc.mesh
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.rebuild()
    ch = C.c_void_p()
    _lib.check(_lib.lib.rq_channel_create(bvh.handle, 2, 128, C.byref(ch)))
    packets = _packets(mesh, 6, [128, 33])
    v0 = mesh.vertices.copy()
    for k in range(4):
        if k == 3:
            bvh.rebuild()
        elif k:
            mesh.vertices = scenes.animated_vertices(v0, k, amplitude=0.05)
            bvh.update(rotate=True)
        for o, d, tm, fl in packets:
            rc, got = _trace(_lib.lib.rq_channel_trace, ch, o, d, tm, fl)
            assert rc == _lib.RQ_OK
            assert _same(got, _trace(_lib.lib.rq_trace, bvh.handle, o, d, tm, fl)[1]), k
    assert _stats(ch)[2] >= 4
    # the scene goes away first: the channel reports it instead of tracing
    h = bvh.handle
    bvh.close()
    o, d, tm, fl = packets[0]
    rc, _ = _trace(_lib.lib.rq_channel_trace, ch, o, d, tm, fl)
    assert rc == _lib.RQ_ERR_STATE
    _lib.check(_lib.lib.rq_channel_destroy(ch))
    del h


def test_channel_arguments(scene):
    from rfmanta_b200 import _lib
    sc, bvh = scene
    ch = C.c_void_p()
    assert _lib.lib.rq_channel_create(None, 4, 64, C.byref(ch)) == _lib.RQ_ERR_ARG
    assert _lib.lib.rq_channel_create(bvh.handle, 5000, 64, C.byref(ch)) == _lib.RQ_ERR_ARG
    assert _lib.lib.rq_channel_create(bvh.handle, 4, 1 << 20, C.byref(ch)) == _lib.RQ_ERR_ARG
    _lib.check(_lib.lib.rq_channel_create(bvh.handle, 0, 0, C.byref(ch)))  # defaults
    o = np.zeros((3, 4), np.float32)
    tm = np.ones(4, np.float32)
    assert _lib.lib.rq_channel_trace(ch, 4, _p(o), _p(o), _p(tm), 7, None, None, None,
                                     None) == _lib.RQ_ERR_ARG
    assert _lib.lib.rq_channel_trace(ch, 4, None, _p(o), _p(tm), 0, None, None, None,
                                     None) == _lib.RQ_ERR_ARG
    assert _lib.lib.rq_channel_trace(ch, 0, None, None, None, 0, None, None, None,
                                     None) == _lib.RQ_OK
    assert _lib.lib.rq_channel_set_timing(ch, 0.0, 1.0, 1.0) == _lib.RQ_ERR_ARG
    assert _stats(ch)[2] == 0  # nothing traced: no kernel was started
    _lib.check(_lib.lib.rq_channel_destroy(ch))


def test_python_mirror_resident_mode(scene):
    """GpuDynBVH.setPacketMode(Resident) (the mirror of the C++ drop-in's
    packet mode) gives intersect() the same results as per-call tracing,
    from several threads at once."""
    import threading
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH, RayBatch
    sc, _ = scene
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    lo, hi = sc.mesh.bounds()
    batches = []
    for k in range(32):
        o, d, tm, _ = scenes.random_rays(64 if k % 4 else 2000, lo - 0.3, hi + 0.3,
                                         seed=700 + k, anyhit_fraction=1.0 if k % 2 else 0.0)
        batches.append((o, d, tm if k % 2 else np.full(tm.shape, 1e19, np.float32), k % 2))
    want = []
    for o, d, tm, a in batches:
        r = RayBatch(o, d, tm, flags=RayBatch.AnyHit if a else 0)
        bvh.intersect(r)
        want.append(r)
    bvh.setPacketMode(GpuDynBVH.Resident)
    got = [None] * len(batches)

    def worker(w):
        for k in range(w, len(batches), 4):
            o, d, tm, a = batches[k]
            r = RayBatch(o, d, tm, flags=RayBatch.AnyHit if a else 0)
            bvh.intersect(r)
            got[k] = r

    th = [threading.Thread(target=worker, args=(w,)) for w in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for g, w in zip(got, want):
        assert np.array_equal(g.hitPrim, w.hitPrim)
        assert np.array_equal(g.minT.view(np.uint32), w.minT.view(np.uint32))
    bvh.setPacketMode(GpuDynBVH.PerCall)
    bvh.close()


def test_channel_wait_is_bounded(scene):
    """The host's wait for a packet is bounded: with a timeout far below a
    PCIe round trip the call returns RQ_ERR_TIMEOUT and retires its slot
    (the device may still answer into it later); once every slot is
    retired the channel reports RQ_ERR_STATE, and a new channel traces
    normally.  No device wait is involved: the kernel itself exits on its
    idle limit."""
    from rfmanta_b200 import _lib
    sc, bvh = scene
    ch = C.c_void_p()
    _lib.check(_lib.lib.rq_channel_create(bvh.handle, 2, 64, C.byref(ch)))
    o, d, tm, fl = _packets(sc.mesh, 1, [64], seed0=900)[0]
    rc, _ = _trace(_lib.lib.rq_channel_trace, ch, o, d, tm, fl)  # kernel up
    assert rc == _lib.RQ_OK
    _lib.check(_lib.lib.rq_channel_set_timing(ch, 20.0, 10.0, 1e-9))
    for _ in range(2):
        rc, _ = _trace(_lib.lib.rq_channel_trace, ch, o, d, tm, fl)
        assert rc == _lib.RQ_ERR_TIMEOUT
    rc, _ = _trace(_lib.lib.rq_channel_trace, ch, o, d, tm, fl)
    assert rc == _lib.RQ_ERR_STATE
    _lib.check(_lib.lib.rq_channel_destroy(ch))
    _lib.check(_lib.lib.rq_channel_create(bvh.handle, 2, 64, C.byref(ch)))
    rc, got = _trace(_lib.lib.rq_channel_trace, ch, o, d, tm, fl)
    assert rc == _lib.RQ_OK and _same(got, _trace(_lib.lib.rq_trace, bvh.handle, o, d, tm, fl)[1])
    _lib.check(_lib.lib.rq_channel_destroy(ch))
