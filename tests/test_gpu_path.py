"""Path-tracing wavefront against its CPU restatement.

Every path draws from its own PCG32 stream and the device keeps the
restatement's float operation order, so the image, the ray counts and the
triangle id of every bounce of every path are compared bit for bit.  The
bounce rays the device produced are also re-traced by the restatement (the
per-bounce intersection parity of the path)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _tree_of(bvh):
    from oracle.pyoracle import Tree
    from rfmanta_b200.treeio import parse_dynbvh_blob
    t = parse_dynbvh_blob(bvh.exportBlob())
    return Tree(t.bounds, t.child, t.children, t.axis, t.left_cheaper, t.ids)


@pytest.fixture(scope="module", params=[0, 1])
def tiny(request):
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.tiny_path_scene()
    bvh = GpuDynBVH(tri_kind=request.param)
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    return request.param, sc, bvh, _tree_of(bvh)


def test_image_and_bounces_bit_exact(tiny, restatement):
    import torch
    kind, sc, bvh, tree = tiny
    n = sc.xres * sc.yres * sc.spp
    D = sc.max_depth
    prim = torch.full((D * n,), -2, dtype=torch.int32, device="cuda")
    org = torch.zeros(3 * D * n, device="cuda")
    dir = torch.zeros(3 * D * n, device="cuda")
    bvh.set_path_debug(prim.data_ptr(), org.data_ptr(), dir.data_ptr(), n)
    out = bvh.render_path(sc)
    bvh.set_path_debug(0, 0, 0, 0)
    exp = restatement.render_path(tree, sc, tri_kind=kind, debug=True)
    gp = prim.cpu().numpy().reshape(D, n)
    assert np.array_equal(gp, exp["prim"])
    assert out["rays"] == exp["rays"] and out["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))
    # re-trace every device bounce ray on the CPU
    o = org.cpu().numpy().reshape(3, D, n)
    d = dir.cpu().numpy().reshape(3, D, n)
    for depth in range(D):
        live = gp[depth] != -2
        if not live.any():
            continue
        oo = np.ascontiguousarray(o[:, depth, live])
        dd = np.ascontiguousarray(d[:, depth, live])
        r = restatement.trace(tree, sc.mesh, oo, dd, np.full(oo.shape[1], 1e19, np.float32),
                              tri_kind=kind)
        assert np.array_equal(r["prim"], gp[depth, live])


def test_chunking_does_not_change_results(tiny):
    kind, sc, bvh, tree = tiny
    a = bvh.render_path(sc)
    b = bvh.render_path(sc, chunk_paths=sc.spp * 37)  # uneven chunks of 37 pixels
    assert np.array_equal(_bits(a["rgb"]), _bits(b["rgb"]))
    assert a["rays"] == b["rays"] and a["shadow_rays"] == b["shadow_rays"]


def test_device_entry_matches_host_entry(tiny):
    import torch
    kind, sc, bvh, tree = tiny
    a = bvh.render_path(sc)
    p = bvh.path_params(sc)
    rgb = torch.zeros(sc.xres * sc.yres * 3, device="cuda")
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    bvh.render_path_device(p, rgb.data_ptr(), cnt.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(_bits(rgb.cpu().numpy().reshape(-1, 3)), _bits(a["rgb"]))
    assert int(cnt[0]) == a["rays"]


def test_medium_frame_sampled_paths(restatement):
    """1.2M-triangle scene at reduced resolution: a sample of pixels is
    compared against the restatement (full radiance per pixel)."""
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.path_scene(xres=160, yres=90, spp=4)
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    tree = _tree_of(bvh)
    out = bvh.render_path(sc)
    for pix0 in (0, 5000, 14000):
        exp = restatement.render_path(tree, sc, paths=(pix0 * sc.spp, (pix0 + 40) * sc.spp))
        r = exp["rad"].reshape(-1, sc.spp, 3)
        acc = np.zeros((r.shape[0], 3), np.float32)
        for s in range(sc.spp):
            acc = (acc + r[:, s]).astype(np.float32)
        acc = (acc * np.float32(1.0 / sc.spp)).astype(np.float32)
        assert np.array_equal(_bits(out["rgb"][pix0:pix0 + 40]), _bits(acc))


@pytest.mark.parametrize("max_depth", [2, 4])
def test_ambient_at_max_depth_bit_exact(tiny, restatement, max_depth):
    """With a ConstantAmbient light the paths that reach their last bounce
    add ambient * kd times their importance (do_ambient_on_maxdepth):
    device and restatement agree bit for bit, in a served request too."""
    import dataclasses
    from rfmanta_b200.serve import RenderServer, request_for_scene
    kind, sc, bvh, tree = tiny
    s2 = dataclasses.replace(sc, ambient=(0.3, 0.4, 0.5), max_depth=max_depth)
    out = bvh.render_path(s2)
    exp = restatement.render_path(tree, s2, tri_kind=kind)
    assert out["rays"] == exp["rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))
    plain = bvh.render_path(dataclasses.replace(s2, ambient=(0.0, 0.0, 0.0)))
    assert np.all(out["rgb"].sum(0) > plain["rgb"].sum(0))
    srv = RenderServer([bvh], path_capacity=1 << 15, chunk_pixels=300)
    q = request_for_scene(0, sc.mesh, s2.xres, s2.yres, s2.spp, max_depth, seed=s2.seed)
    q = dataclasses.replace(q, eye=s2.camera.eye, lookat=s2.camera.lookat, up=s2.camera.up,
                            hfov=s2.camera.hfov, vfov=s2.camera.vfov, rr_depth=s2.rr_depth,
                            light_anchor=s2.light.anchor, light_v1=s2.light.v1,
                            light_v2=s2.light.v2, light_color=s2.light.color,
                            background=s2.background, ambient=s2.ambient,
                            materials=sc.mesh.materials)
    rid = srv.submit(q)
    for _ in range(10000):
        srv.step()
        if rid in srv.poll():
            break
    img, _, _ = srv.result(rid, q.xres, q.yres)
    srv.close()
    assert np.array_equal(_bits(img), _bits(out["rgb"]))


@pytest.mark.parametrize("regs", [(1, 1), (2, 2), (4, 4), (4, 0), (0, 2)])
def test_register_stack_entries_do_not_change_results(tiny, restatement, regs):
    """The persistent stages keep 0, 1, 2 or 4 of the newest traversal-stack
    entries in registers (the rest in the thread's shared-memory column);
    image, ray counts and per-bounce ids are those of the restatement
    whatever the split, also in a block shape with a small column."""
    from rfmanta_b200._lib import RQ_PATH_EXTEND, RQ_PATH_SHADE
    kind, sc, bvh, tree = tiny
    old = [bvh.get_launch_config(False, stage=s) for s in (RQ_PATH_EXTEND, RQ_PATH_SHADE)]
    try:
        for stage, r in zip((RQ_PATH_EXTEND, RQ_PATH_SHADE), regs):
            bvh.set_launch_config(False, block_threads=64, refill_threshold=8, stage=stage,
                                  reg_stack=r)
        out = bvh.render_path(sc)
    finally:
        for stage, c in zip((RQ_PATH_EXTEND, RQ_PATH_SHADE), old):
            bvh.set_launch_config(False, stage=stage, **c)
    exp = restatement.render_path(tree, sc, tri_kind=kind)
    assert out["rays"] == exp["rays"] and out["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))


def test_register_stack_entries_rejected_outside_0_1_2_4(tiny):
    from rfmanta_b200._lib import RQ_PATH_EXTEND, RQError
    kind, sc, bvh, tree = tiny
    with pytest.raises(RQError):
        bvh.set_launch_config(False, stage=RQ_PATH_EXTEND, reg_stack=3)


@pytest.mark.parametrize("layout", [1, 2])
def test_node_layouts_do_not_change_results(tiny, restatement, layout):
    """The path stages can read a breadth-first (1) or hot-top (2) copy of
    the node records; the records and the traversal order are unchanged, so
    image, ray counts and per-bounce ids stay those of the restatement."""
    from rfmanta_b200._lib import RQ_PATH_EXTEND
    kind, sc, bvh, tree = tiny
    old = bvh.get_launch_config(False, stage=RQ_PATH_EXTEND)
    try:
        bvh.set_launch_config(False, stage=RQ_PATH_EXTEND,
                              **dict(old, node_layout=layout))
        out = bvh.render_path(sc)
    finally:
        bvh.set_launch_config(False, stage=RQ_PATH_EXTEND, **old)
    exp = restatement.render_path(tree, sc, tri_kind=kind)
    assert out["rays"] == exp["rays"] and out["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))


def test_path_image_into_page_locked_host_memory(tiny):
    """An image given in page-locked host memory equals the image copied
    to pageable memory, with the same ray counts."""
    import ctypes as C
    import torch
    from rfmanta_b200 import _lib
    kind, sc, bvh, tree = tiny
    want = bvh.render_path(sc)
    rgb = torch.empty((sc.xres * sc.yres, 3), pin_memory=True)
    counts = (C.c_uint64 * 2)()
    p = bvh.path_params(sc)
    _lib.check(_lib.lib.rq_render_path(bvh.handle, C.byref(p), C.c_void_p(rgb.data_ptr()), counts))
    assert counts[0] == want["rays"] and counts[1] == want["shadow_rays"]
    assert np.array_equal(rgb.numpy().view(np.uint32), want["rgb"].view(np.uint32))
