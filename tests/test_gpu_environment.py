"""EyeAmbient and LinearBackground on the device (rq_environment): every
frame entry point against the reference's fixture (tests/golden/
tiny_env.npz) or the CPU restatement, bit for bit, and the argument checks."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _env(ambient="eye", background="linear"):
    from rfmanta_b200 import scenes
    return scenes.Environment(ambient=ambient, background=background,
                              background_down=(0.9, 0.3, 0.1), background_up=(0.2, 1.0, 0.3))


@pytest.fixture(scope="module")
def env_case():
    from rfmanta_b200.dynbvh import GpuDynBVH
    from test_oracle_environment import env_tree, load_env, whitted_case
    g = load_env()
    sc = whitted_case()
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.importTree(env_tree(g))
    return g, sc, bvh


def test_whitted_entry_points_match_reference_fixture(env_case):
    import torch
    from rfmanta_b200 import _lib
    g, sc, bvh = env_case
    out = bvh.render_whitted(sc)
    assert out["shadow_rays"] == int(g["whitted_shadow_rays"])
    assert np.array_equal(out["prim"], g["whitted_prim"])
    assert np.array_equal(_bits(out["rgb"]), _bits(g["whitted_rgb"]))
    # the supersampled frame at 1 spp and the no-allocation entry point
    f = dataclasses.replace(sc)
    f.spp, f.seed = 1, 0
    assert np.array_equal(_bits(bvh.render_frame(f)["rgb"]), _bits(g["whitted_rgb"]))
    p = bvh.whitted_params(sc)
    npx = sc.xres * sc.yres
    rgb = torch.zeros(npx * 3, device="cuda")
    t = torch.zeros(npx, device="cuda")
    prim = torch.zeros(npx, dtype=torch.int32, device="cuda")
    ns = torch.zeros(1, dtype=torch.int64, device="cuda")
    _lib.check(_lib.lib.rq_render_whitted_device_noalloc(
        bvh.handle, C.byref(p), C.c_void_p(rgb.data_ptr()), C.c_void_p(t.data_ptr()),
        C.c_void_p(prim.data_ptr()), C.c_void_p(ns.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    assert np.array_equal(_bits(rgb.cpu().numpy().reshape(-1, 3)), _bits(g["whitted_rgb"]))


def test_reflective_frame_matches_reference_fixture(env_case):
    import os
    import sys
    from conftest import GOLDEN
    sys.path.insert(0, GOLDEN)
    from make_golden import REFLECT
    from test_gpu_instance import _pixels_from_samples
    g, sc, bvh = env_case
    f = dataclasses.replace(sc)
    f.xres, f.yres, f.spp, f.seed = 40, 32, 4, 5
    n = f.mesh.materials.shape[0]
    f.specular = np.full((n, 3), 0.4, np.float32)
    f.specpow = np.array(REFLECT["flat_specpow"][:n], np.int32)
    f.reflectivity = np.array(REFLECT["flat_refl"][:n], np.float32)
    out = bvh.render_frame(f)
    assert out["shadow_rays"] == int(g["frame_shadow_rays"])
    assert np.array_equal(_bits(out["rgb"]),
                          _bits(_pixels_from_samples(g["frame_sample_rgb"], f.spp)))


@pytest.mark.parametrize("ambient,background", [("eye", "linear"), ("eye", "constant"),
                                                ("constant", "linear")])
def test_two_level_frame_matches_restatement(restatement, ambient, background):
    from test_gpu_instance import _device_scene
    from test_oracle_instance import golden_world, load_instanced, tiny_scene_from_golden
    g = load_instanced()
    top, inner = _device_scene(g)
    sc = tiny_scene_from_golden(g)
    sc.environment = _env(ambient, background)
    out = top.render_frame(sc, g["materials"])
    W = golden_world(restatement, g)
    exp = restatement.render_frame(W, sc, g["materials"], specular=g["specular"],
                                   specpow=g["specpow"])
    assert out["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("max_depth", [1, 2, 4])
def test_path_bit_exact_and_served(restatement, kind, max_depth):
    """The path tracer with EyeAmbient (at the last bounce, against the
    sampled direction) and LinearBackground (on every miss): device and
    restatement agree bit for bit, and a served request equals the frame."""
    from test_gpu_path import _tree_of
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    from rfmanta_b200.serve import RenderServer, request_for_scene
    sc = scenes.tiny_path_scene()
    sc = dataclasses.replace(sc, ambient=(0.3, 0.4, 0.5), max_depth=max_depth,
                             environment=_env())
    bvh = GpuDynBVH(tri_kind=kind)
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    tree = _tree_of(bvh)
    out = bvh.render_path(sc)
    exp = restatement.render_path(tree, sc, tri_kind=kind)
    assert out["rays"] == exp["rays"] and out["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))
    plain = bvh.render_path(dataclasses.replace(sc, environment=None))
    assert not np.array_equal(plain["rgb"], out["rgb"])
    srv = RenderServer([bvh], path_capacity=1 << 15, chunk_pixels=300)
    q = request_for_scene(0, sc.mesh, sc.xres, sc.yres, sc.spp, max_depth, seed=sc.seed)
    q = dataclasses.replace(q, eye=sc.camera.eye, lookat=sc.camera.lookat, up=sc.camera.up,
                            hfov=sc.camera.hfov, vfov=sc.camera.vfov, rr_depth=sc.rr_depth,
                            light_anchor=sc.light.anchor, light_v1=sc.light.v1,
                            light_v2=sc.light.v2, light_color=sc.light.color,
                            background=sc.background, ambient=sc.ambient,
                            materials=sc.mesh.materials, environment=sc.environment)
    rid = srv.submit(q)
    for _ in range(10000):
        srv.step()
        if rid in srv.poll():
            break
    img, _, _ = srv.result(rid, q.xres, q.yres)
    srv.close()
    assert np.array_equal(_bits(img), _bits(out["rgb"]))


def test_bad_environment_is_refused(env_case):
    from rfmanta_b200 import _lib, scenes
    from rfmanta_b200.serve import RenderServer, request_for_scene
    g, sc, bvh = env_case
    bad = [scenes.Environment(background="linear", background_up=(0.0, 0.0, 0.0))]
    for env in bad:
        s = dataclasses.replace(sc, environment=env)
        with pytest.raises(RuntimeError):
            bvh.render_whitted(s)
    p = bvh.whitted_params(sc)
    p.environment.ambient_kind = 7
    rgb = np.zeros((sc.xres * sc.yres, 3), np.float32)
    rc = _lib.lib.rq_render_whitted(bvh.handle, C.byref(p), rgb.ctypes.data_as(C.c_void_p),
                                    None, None, None)
    assert rc == _lib.RQ_ERR_ARG
    srv = RenderServer([bvh], path_capacity=1 << 15, chunk_pixels=300)
    q = request_for_scene(0, sc.mesh, 16, 16, 1, 1, seed=1)
    q.environment = scenes.Environment(background="linear", background_up=(0.0, 0.0, 0.0))
    with pytest.raises(RuntimeError):
        srv.submit(q)
    srv.close()
