"""The submission queue (rq_queue_*): many host threads each tracing small
packets and waiting for them, the way Manta's render workers call
DynBVH::intersect.  Every packet's results equal rq_trace's on the same
rays, bit for bit, whether it went out alone or gathered with others, for
closest and any hit; packets larger than the batch capacity go through
rq_trace; the queue gathers packets when threads wait concurrently."""
import ctypes as C
import threading

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


def test_queue_matches_plain_trace_across_threads():
    from rfmanta_b200 import _lib, scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.small_frame_scene(level=5, grid=60)
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    q = C.c_void_p()
    _lib.check(_lib.lib.rq_queue_create(bvh.handle, 64 * 32, C.byref(q)))
    lo, hi = sc.mesh.bounds()
    packets = []
    for k in range(48 * 12):
        n = [64, 1, 37, 64, 5][k % 5]
        any_ = k % 3 == 0
        o, d, tm, _ = scenes.random_rays(n, lo - 0.3, hi + 0.3, seed=k,
                                         anyhit_fraction=1.0 if any_ else 0.0)
        if not any_:
            tm = np.full(n, 1e19, np.float32)
        packets.append((np.ascontiguousarray(o), np.ascontiguousarray(d),
                        np.ascontiguousarray(tm), _lib.RQ_ANYHIT if any_ else _lib.RQ_CLOSEST))
    # one oversized packet (beyond the batch capacity) too
    o, d, _, _ = scenes.random_rays(5000, lo - 0.3, hi + 0.3, seed=999)
    packets.append((np.ascontiguousarray(o), np.ascontiguousarray(d),
                    np.full(5000, 1e19, np.float32), _lib.RQ_CLOSEST))
    results = [None] * len(packets)
    errors = []

    def worker(w):
        for k in range(w, len(packets), 48):
            o, d, tm, fl = packets[k]
            rc, out = _trace(_lib.lib.rq_queue_trace, q, o, d, tm, fl)
            if rc != _lib.RQ_OK:
                errors.append((k, rc))
            results[k] = out

    th = [threading.Thread(target=worker, args=(w,)) for w in range(48)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for k, (o, d, tm, fl) in enumerate(packets):
        rc, want = _trace(_lib.lib.rq_trace, bvh.handle, o, d, tm, fl)
        assert rc == _lib.RQ_OK
        got = results[k]
        assert np.array_equal(got["prim"], want["prim"]), k
        if fl == _lib.RQ_CLOSEST:
            for f in ("t", "u", "v"):
                assert np.array_equal(got[f].view(np.uint32), want[f].view(np.uint32)), (k, f)
    b, p, r = C.c_longlong(), C.c_longlong(), C.c_longlong()
    _lib.check(_lib.lib.rq_queue_stats(q, C.byref(b), C.byref(p), C.byref(r)))
    assert p.value == len(packets) - 1  # the oversized packet bypasses the queue
    assert 0 < b.value <= p.value
    _lib.lib.rq_queue_destroy(q)
