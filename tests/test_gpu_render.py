"""Device Whitted frame (raygen + closest hit + compaction, fused Lambertian
shading with hard-shadow any-hit) against the reference's frame and the CPU
restatement.  Colours, distances and triangle ids are compared bit for bit;
the largest per-channel difference is reported as well (0 expected)."""
import numpy as np
import pytest

from conftest import golden_mesh, golden_tree

pytestmark = pytest.mark.gpu

KIND = {"wald": 0, "ks": 1}


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _scene_from_golden(g):
    from rfmanta_b200.scenes import Camera, PointLightSpec, WhittedScene
    c = g["cam"]
    cam = Camera(tuple(c[0:3]), tuple(c[3:6]), tuple(c[6:9]), float(c[9]), float(c[10]))
    lights = [PointLightSpec(tuple(l[:3]), tuple(l[3:])) for l in g["lights"]]
    return WhittedScene(golden_mesh(g), cam, lights, tuple(g["ambient"]),
                        tuple(g["background"]), int(g["xres"]), int(g["yres"]))


def test_golden_frame(golden):
    from rfmanta_b200.dynbvh import GpuDynBVH
    kind, g = golden
    sc = _scene_from_golden(g)
    bvh = GpuDynBVH(tri_kind=KIND[kind])
    bvh.setGroup(sc.mesh)
    bvh.importTree(golden_tree(g))
    out = bvh.render_whitted(sc)
    assert out["shadow_rays"] == int(g["img_shadow_rays"])
    assert np.array_equal(out["prim"], g["img_prim"])
    assert np.array_equal(_bits(out["t"]), _bits(g["img_t"]))
    err = np.abs(out["rgb"] - g["img_rgb"]).max()
    assert err == 0.0, f"max per-channel error {err}"
    assert np.array_equal(_bits(out["rgb"]), _bits(g["img_rgb"]))


def test_small_frame_matches_restatement(restatement):
    """Full 512x512 frame over ~102k triangles, one point light."""
    from oracle.pyoracle import Reference
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    if not Reference.available():
        pytest.skip("needs a reference-built tree")
    sc = scenes.small_frame_scene()
    for kind in (0, 1):
        tree = Reference().scene(sc.mesh, kind).tree()
        bvh = GpuDynBVH(tri_kind=kind)
        bvh.setGroup(sc.mesh)
        bvh.importTree(tree)
        out = bvh.render_whitted(sc)
        exp = restatement.render_whitted(tree, sc, tri_kind=kind)
        assert out["shadow_rays"] == exp["shadow_rays"]
        assert np.array_equal(out["prim"], exp["prim"])
        assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))


def test_render_device_path_matches_host_path(golden):
    import torch
    from rfmanta_b200.dynbvh import GpuDynBVH
    kind, g = golden
    sc = _scene_from_golden(g)
    bvh = GpuDynBVH(tri_kind=KIND[kind])
    bvh.setGroup(sc.mesh)
    bvh.importTree(golden_tree(g))
    npx = sc.xres * sc.yres
    rgb = torch.zeros(npx * 3, device="cuda")
    t = torch.zeros(npx, device="cuda")
    prim = torch.zeros(npx, dtype=torch.int32, device="cuda")
    ns = torch.zeros(1, dtype=torch.int64, device="cuda")
    p = bvh.whitted_params(sc)
    for _ in range(2):  # a second frame reuses the scratch and counters
        bvh.render_whitted_device(p, rgb.data_ptr(), t.data_ptr(), prim.data_ptr(),
                                  ns.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert int(ns.item()) == int(g["img_shadow_rays"])
        assert np.array_equal(_bits(rgb.cpu().numpy().reshape(-1, 3)), _bits(g["img_rgb"]))


def test_frames_into_page_locked_host_memory():
    """Frame outputs given in page-locked host memory (as the bench's
    end-to-end runs give them) equal those written to pageable memory bit
    for bit, for the Whitted frame and the supersampled frame, with and
    without the optional t / prim outputs."""
    import ctypes as C
    import torch
    from rfmanta_b200 import _lib, scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.small_frame_scene(level=4, grid=40, xres=200, yres=150)
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    npx = sc.xres * sc.yres
    want = bvh.render_whitted(sc)
    rgb = torch.empty((npx, 3), pin_memory=True)
    t = torch.empty(npx, pin_memory=True)
    prim = torch.empty(npx, dtype=torch.int32, pin_memory=True)
    ns = C.c_uint64()
    p = bvh.whitted_params(sc)
    _lib.check(_lib.lib.rq_render_whitted(bvh.handle, C.byref(p), C.c_void_p(rgb.data_ptr()),
                                          C.c_void_p(t.data_ptr()), C.c_void_p(prim.data_ptr()),
                                          C.byref(ns)))
    assert ns.value == want["shadow_rays"]
    assert np.array_equal(prim.numpy(), want["prim"])
    assert np.array_equal(t.numpy().view(np.uint32), want["t"].view(np.uint32))
    assert np.array_equal(rgb.numpy().view(np.uint32), want["rgb"].view(np.uint32))
    # only the image pinned, t and prim not wanted
    rgb2 = torch.empty((npx, 3), pin_memory=True)
    _lib.check(_lib.lib.rq_render_whitted(bvh.handle, C.byref(p), C.c_void_p(rgb2.data_ptr()),
                                          None, None, None))
    assert np.array_equal(rgb2.numpy().view(np.uint32), want["rgb"].view(np.uint32))
    # the supersampled frame
    sc.spp, sc.seed = 4, 11
    fw = bvh.render_frame(sc, sc.mesh.materials)
    fp = bvh.frame_params(sc, sc.mesh.materials)
    rgb3 = torch.empty((npx, 3), pin_memory=True)
    _lib.check(_lib.lib.rq_render_frame(bvh.handle, C.byref(fp), C.c_void_p(rgb3.data_ptr()),
                                        C.byref(ns)))
    assert ns.value == fw["shadow_rays"]
    assert np.array_equal(rgb3.numpy().view(np.uint32), fw["rgb"].view(np.uint32))
