"""Continuous-batching server: each request's image is the same bits alone
and in a mix of requests of other scenes, sizes, spp and depths; equal to
the single-frame path tracer for the same parameters; admission respects
the HBM budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def scenes3():
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    meshes = [scenes.tiny_path_scene().mesh, scenes.sphere_set(4, 3, seed=2),
              scenes.heightfield(30, 30, seed=3, extent=4.0, y=0.0)]
    meshes[2].materials = np.array([[0.6, 0.5, 0.4]], np.float32)
    bvhs = []
    for m in meshes:
        b = GpuDynBVH()
        b.setGroup(m)
        b.rebuild()
        bvhs.append(b)
    return meshes, bvhs


def _requests(meshes):
    from rfmanta_b200.serve import request_for_scene
    spec = [(0, 40, 30, 4, 4), (1, 64, 48, 1, 1), (2, 33, 17, 16, 3), (0, 90, 60, 1, 5),
            (1, 20, 20, 4, 2), (2, 128, 72, 4, 4), (0, 7, 5, 16, 4), (1, 50, 40, 9, 3)]
    return [request_for_scene(s, meshes[s], x, y, spp, d, seed=50 + i)
            for i, (s, x, y, spp, d) in enumerate(spec)]


def _run(server, reqs):
    ids = [server.submit(r) for r in reqs]
    out = {}
    for _ in range(100000):
        server.step()
        for rid in server.poll():
            i = ids.index(rid)
            img, lat, _ = server.result(rid, reqs[i].xres, reqs[i].yres)
            out[i] = img
            server.release(rid)
        if len(out) == len(reqs):
            return [out[i] for i in range(len(reqs))]
    raise AssertionError("server did not finish")


def test_alone_equals_mixed(scenes3):
    from rfmanta_b200.serve import RenderServer
    meshes, bvhs = scenes3
    reqs = _requests(meshes)
    alone = []
    for r in reqs:
        srv = RenderServer(bvhs, path_capacity=1 << 16, chunk_pixels=1000)
        alone.append(_run(srv, [r])[0])
        srv.close()
    srv = RenderServer(bvhs, path_capacity=1 << 16, chunk_pixels=1000)
    mixed = _run(srv, reqs)
    st = srv.stats()
    assert st["steps"] > 1 and st["rays"] > 0
    srv.close()
    for a, m in zip(alone, mixed):
        assert np.array_equal(_bits(a), _bits(m))


def test_server_equals_frame_path_tracer(scenes3):
    from rfmanta_b200 import scenes
    from rfmanta_b200.serve import RenderServer
    meshes, bvhs = scenes3
    r = _requests(meshes)[0]
    srv = RenderServer(bvhs, path_capacity=1 << 15, chunk_pixels=333)
    img = _run(srv, [r])[0]
    srv.close()
    ps = scenes.PathScene(meshes[0], scenes.Camera(r.eye, r.lookat, r.up, r.hfov, r.vfov),
                          scenes.AreaLightSpec(r.light_anchor, r.light_v1, r.light_v2,
                                               r.light_color),
                          r.background, r.xres, r.yres, r.spp, r.max_depth, r.rr_depth, r.seed)
    ref = bvhs[0].render_path(ps)
    assert np.array_equal(_bits(img), _bits(ref["rgb"]))


def test_admission_waits_for_budget(scenes3):
    from rfmanta_b200 import _lib
    from rfmanta_b200.serve import RenderServer
    meshes, bvhs = scenes3
    reqs = _requests(meshes)[:4]
    big = max(r.xres * r.yres * 12 for r in reqs)
    srv = RenderServer(bvhs, path_capacity=1 << 16, chunk_pixels=1000,
                       hbm_budget_bytes=big + 64)
    for r in reqs:
        srv.submit(r)
    srv.step()
    st = srv.stats()
    assert st["active"] + st["pending"] == 4 and st["pending"] >= 1
    assert st["bytes_in_use"] <= big + 64
    srv.close()
    srv = RenderServer(bvhs, path_capacity=1 << 16, chunk_pixels=1000, hbm_budget_bytes=1000)
    with pytest.raises(_lib.RQError) as e:
        srv.submit(reqs[3])
    assert e.value.code == _lib.RQ_ERR_CAPACITY
    srv.close()


def test_server_follows_scene_updates():
    """A server keeps serving a scene whose mesh moved (rotating update,
    new layout, possibly a deeper tree): the next step copies in the new
    descriptor, and a request after the update equals the frame path
    tracer on the updated scene."""
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    from rfmanta_b200.serve import RenderServer, request_for_scene
    mesh = scenes.tiny_path_scene().mesh
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.rebuild()
    srv = RenderServer([bvh], path_capacity=1 << 15, chunk_pixels=500)
    r = request_for_scene(0, mesh, 40, 30, 4, 4, seed=7)
    _run(srv, [r])
    v0 = mesh.vertices.copy()
    for k in (1, 2):
        mesh.vertices = scenes.animated_vertices(v0, k, amplitude=0.05)
        bvh.update()
        img = _run(srv, [r])[0]
        ps = scenes.PathScene(mesh, scenes.Camera(r.eye, r.lookat, r.up, r.hfov, r.vfov),
                              scenes.AreaLightSpec(r.light_anchor, r.light_v1, r.light_v2,
                                                   r.light_color),
                              r.background, r.xres, r.yres, r.spp, r.max_depth, r.rr_depth,
                              r.seed)
        assert np.array_equal(_bits(img), _bits(bvh.render_path(ps)["rgb"]))
    srv.close()


def test_ray_queries_beside_renders(scenes3):
    """Ray-query requests (closest and any hit, 1 to 2.5M rays, beyond one
    step's 8Mi-ray budget in total) are served in the same steps as render
    requests: every query's t and triangle ids equal rq_trace on the same
    rays, and every render equals the same request rendered alone."""
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import RayBatch
    from rfmanta_b200.serve import RenderServer
    meshes, bvhs = scenes3
    reqs = _requests(meshes)[:4]
    queries = []
    for k, (si, n, anyhit) in enumerate([(0, 1, False), (1, 5000, True), (2, 2_500_000, False),
                                         (0, 300_000, True), (1, 2_600_000, False),
                                         (2, 3_100_000, True)]):
        lo, hi = meshes[si].bounds()
        o, d, tm, _ = scenes.random_rays(n, lo - 0.2, hi + 0.2, seed=900 + k,
                                         anyhit_fraction=1.0 if anyhit else 0.0)
        if not anyhit:
            tm = np.full(n, 1e19, np.float32)
        queries.append((si, o, d, tm, anyhit))
    srv = RenderServer(bvhs, path_capacity=1 << 16, chunk_pixels=1000)
    alone = _run(srv, reqs)
    srv.close()
    srv = RenderServer(bvhs, path_capacity=1 << 16, chunk_pixels=1000)
    rids, qids = [], []
    for i in range(max(len(reqs), len(queries))):
        if i < len(queries):
            si, o, d, tm, anyhit = queries[i]
            qids.append(srv.submit_query(si, o, d, tm, anyhit))
        if i < len(reqs):
            rids.append(srv.submit(reqs[i]))
    imgs, qres = {}, {}
    for _ in range(100000):
        srv.step()
        for rid in srv.poll():
            if rid in qids:
                k = qids.index(rid)
                t, prim, lat, _ = srv.query_result(rid, queries[k][3].shape[0])
                qres[k] = (t, prim)
            else:
                k = rids.index(rid)
                imgs[k], _, _ = srv.result(rid, reqs[k].xres, reqs[k].yres)
            srv.release(rid)
        if len(imgs) == len(reqs) and len(qres) == len(queries):
            break
    st = srv.stats()
    srv.close()
    assert len(imgs) == len(reqs) and len(qres) == len(queries)
    for k in range(len(reqs)):
        assert np.array_equal(_bits(imgs[k]), _bits(alone[k])), k
    for k, (si, o, d, tm, anyhit) in enumerate(queries):
        r = RayBatch(o, d, tm, flags=RayBatch.AnyHit if anyhit else 0)
        bvhs[si].intersect(r)
        t, prim = qres[k]
        if anyhit:
            assert np.array_equal(prim >= 0, r.wasHit()), k
        else:
            assert np.array_equal(prim, r.hitPrim), k
            assert np.array_equal(_bits(t), _bits(r.minT)), k
    assert st["rays"] >= sum(q[1].shape[1] for q in queries)


def test_query_errors(scenes3):
    import ctypes as C
    from rfmanta_b200 import _lib
    from rfmanta_b200.serve import RenderServer
    meshes, bvhs = scenes3
    srv = RenderServer(bvhs, path_capacity=1 << 16, chunk_pixels=1000)
    o = np.zeros((3, 4), np.float32)
    q = _lib.ServeQuery(7, 4, 0, o.ctypes.data, o.ctypes.data, o[0].ctypes.data)
    rid = C.c_int()
    assert _lib.lib.rq_server_submit_query(srv._h, C.byref(q), C.byref(rid)) == _lib.RQ_ERR_ARG
    q.scene, q.flags = 0, 5
    assert _lib.lib.rq_server_submit_query(srv._h, C.byref(q), C.byref(rid)) == _lib.RQ_ERR_ARG
    q.flags = 0
    _lib.check(_lib.lib.rq_server_submit_query(srv._h, C.byref(q), C.byref(rid)))
    # a query's result is not an image, and not ready before it ran
    assert _lib.lib.rq_server_result(srv._h, rid.value, None, None, None) == _lib.RQ_ERR_ARG
    assert _lib.lib.rq_server_query_result(srv._h, rid.value, None, None, None,
                                           None) == _lib.RQ_ERR_STATE
    srv.close()


def test_run_stream_in_the_library(scenes3):
    """rq_server_run_stream: a timed arrival stream submitted, stepped and
    collected inside the library; every image equals the request rendered
    alone by rq_render_path, every request has a latency, and the per-step
    records account for every step and path."""
    from rfmanta_b200 import scenes
    from rfmanta_b200.serve import RenderServer
    meshes, bvhs = scenes3
    reqs = _requests(meshes)
    stream = [(0.002 * i, r) for i, r in enumerate(reqs)]
    srv = RenderServer(bvhs, path_capacity=1 << 16, chunk_pixels=1000)
    srv.set_profile(True)
    b0 = srv.stats()
    out = srv.run_stream(stream, keep_images=True, timeout_s=120.0)
    st = srv.stats()
    prof = srv.profile()
    srv.close()
    assert len(out["info"]) == len(reqs) and out["wall_s"] > 0
    for i, r in enumerate(reqs):
        ps = scenes.PathScene(meshes[r.scene], scenes.Camera(r.eye, r.lookat, r.up, r.hfov, r.vfov),
                              scenes.AreaLightSpec(r.light_anchor, r.light_v1, r.light_v2,
                                                   r.light_color),
                              r.background, r.xres, r.yres, r.spp, r.max_depth, r.rr_depth, r.seed)
        want = bvhs[r.scene].render_path(ps)["rgb"]
        assert np.array_equal(_bits(out["info"][i]["image"]), _bits(want)), i
        assert out["info"][i]["latency"] > 0
    assert len(prof) == st["steps"] - b0["steps"]
    assert sum(p["paths"] for p in prof) == sum(r.xres * r.yres * r.spp for r in reqs)
    assert all(p["gpu_ms"] > 0 for p in prof)
