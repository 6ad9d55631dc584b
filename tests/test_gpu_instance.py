"""Two-level (InstanceT) scenes and the supersampled frame on the device,
bit for bit against the reference fixture (tests/golden/tiny_instanced.npz,
the reference's own trees imported) and against the CPU restatement on
GPU-built trees."""
import numpy as np
import pytest

from test_oracle_instance import golden_world, load_instanced, tiny_scene_from_golden

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _tree(g, name):
    from oracle.pyoracle import Tree
    return Tree(*[g[f"{name}_{f}"] for f in ("bounds", "child", "children", "axis",
                                             "left_cheaper", "ids")])


def _device_scene(g, import_trees=True, tri_kind=0):
    from rfmanta_b200.dynbvh import GpuDynBVH, InstancedBVH
    from rfmanta_b200.scenes import Mesh
    inner = []
    for i in range(int(g["n_inner"])):
        b = GpuDynBVH(tri_kind=tri_kind)
        b.setGroup(Mesh(g[f"inner{i}_vertices"], g[f"inner{i}_indices"],
                        g[f"inner{i}_face_material"], g["materials"]))
        if import_trees:
            b.importTree(_tree(g, f"inner{i}"))
        else:
            b.rebuild()
        inner.append(b)
    top = InstancedBVH(inner, g["inst_scene"], g["translation"], g["kind"])
    top.rebuild()
    if import_trees:
        top.importTree(_tree(g, "top"))
    return top, inner


def _trace(bvh, org, dir, tmax, anyhit):
    import torch
    n = tmax.shape[0]
    d = torch.device("cuda")
    o = torch.from_numpy(np.ascontiguousarray(org)).to(d)
    di = torch.from_numpy(np.ascontiguousarray(dir)).to(d)
    tm = torch.from_numpy(np.ascontiguousarray(tmax)).to(d)
    t = torch.empty(n, dtype=torch.float32, device=d)
    prim = torch.empty(n, dtype=torch.int32, device=d)
    u = torch.empty(n, dtype=torch.float32, device=d)
    v = torch.empty(n, dtype=torch.float32, device=d)
    inst = torch.empty(n, dtype=torch.int32, device=d)
    bvh.intersect_device_ex(n, o.data_ptr(), di.data_ptr(), tm.data_ptr(), anyhit,
                            t.data_ptr(), prim.data_ptr(), u.data_ptr(), v.data_ptr(),
                            inst.data_ptr())
    torch.cuda.synchronize()
    out = dict(t=t.cpu().numpy(), prim=prim.cpu().numpy(), u=u.cpu().numpy(),
               v=v.cpu().numpy(), inst=inst.cpu().numpy())
    out["hit"] = (out["prim"] >= 0).astype(np.int32)
    return out


def test_queries_match_reference_fixture():
    g = load_instanced()
    top, inner = _device_scene(g)
    for tag, anyhit in (("rand", False), ("any", True)):
        org, dir = g[f"{tag}_org"], g[f"{tag}_dir"]
        tmax = g["any_tmax"] if anyhit else np.full(org.shape[1], 1e19, np.float32)
        got = _trace(top, org, dir, tmax, anyhit)
        assert np.array_equal(got["hit"], g[f"{tag}_hit"])
        assert np.array_equal(got["prim"], g[f"{tag}_prim"])
        if not anyhit:
            assert np.array_equal(_bits(got["t"]), _bits(g[f"{tag}_t"]))
            outside = (g[f"{tag}_hit"] == 1) & (g[f"{tag}_inst"] < 0)
            for k in ("u", "v"):
                assert np.array_equal(_bits(got[k])[outside], _bits(g[f"{tag}_{k}"])[outside])
        ihit = g[f"{tag}_inst"] >= 0
        assert np.array_equal(got["inst"][ihit], g[f"{tag}_inst"][ihit])


def test_host_trace_dispatches_two_level():
    from rfmanta_b200.dynbvh import RayBatch
    g = load_instanced()
    top, inner = _device_scene(g)
    rays = RayBatch(g["rand_org"], g["rand_dir"])
    top.intersect(rays)
    assert np.array_equal(rays.hitPrim, g["rand_prim"])
    assert np.array_equal(_bits(rays.minT), _bits(g["rand_t"]))


def test_frame_matches_reference_fixture():
    g = load_instanced()
    top, inner = _device_scene(g)
    sc = tiny_scene_from_golden(g)
    out = top.render_frame(sc, g["materials"])
    r = g["sample_rgb"].reshape(-1, sc.spp, 3)
    acc = np.zeros((r.shape[0], 3), np.float32)
    for s in range(sc.spp):
        acc = (acc + r[:, s]).astype(np.float32)
    exp = (acc * np.float32(np.float32(1.0) / np.float32(sc.spp))).astype(np.float32)
    assert out["shadow_rays"] == int(g["shadow_rays"])
    err = np.abs(out["rgb"] - exp).max()
    assert err == 0.0, f"max per-channel error {err}"
    assert np.array_equal(_bits(out["rgb"]), _bits(exp))


def test_gpu_built_trees_match_restatement(restatement):
    """GPU-built inner and top-level trees, exported and replayed by the
    restatement: queries (t, id, u, v, instance) and the frame agree."""
    from oracle.pyoracle import Tree
    from rfmanta_b200.treeio import parse_dynbvh_blob
    g = load_instanced()
    top, inner = _device_scene(g, import_trees=False)

    def exported(b, n):
        f = parse_dynbvh_blob(b.exportBlob(), n)
        return Tree(f.bounds, f.child, f.children, f.axis, f.left_cheaper, f.ids)
    from rfmanta_b200.scenes import Mesh
    W = restatement.world(
        exported(top, top.n_instances),
        inner=[(exported(b, int(g[f"inner{i}_indices"].shape[0])),
                Mesh(g[f"inner{i}_vertices"], g[f"inner{i}_indices"],
                     g[f"inner{i}_face_material"], g["materials"]))
               for i, b in enumerate(inner)],
        inst_scene=g["inst_scene"], translation=g["translation"], kind=g["kind"])
    for tag, anyhit in (("rand", False), ("any", True)):
        org, dir = g[f"{tag}_org"], g[f"{tag}_dir"]
        tmax = g["any_tmax"] if anyhit else np.full(org.shape[1], 1e19, np.float32)
        got = _trace(top, org, dir, tmax, anyhit)
        exp = restatement.trace_world(W, org, dir, tmax, anyhit)
        assert np.array_equal(got["prim"], exp["prim"])
        assert np.array_equal(got["inst"], exp["inst"])
        if not anyhit:
            for k in ("t", "u", "v"):
                assert np.array_equal(_bits(got[k]), _bits(exp[k])), k
    sc = tiny_scene_from_golden(g)
    out = top.render_frame(sc, g["materials"])
    exp = restatement.render_frame(W, sc, g["materials"], specular=sc.specular,
                                   specpow=sc.specpow)
    assert out["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))


def test_flat_frame_spp1_equals_whitted_frame():
    """rq_render_frame with one sample per pixel is rq_render_whitted."""
    from conftest import golden_mesh, golden_tree, load_golden
    from test_gpu_render import _scene_from_golden
    from rfmanta_b200.dynbvh import GpuDynBVH
    g = load_golden("wald")
    sc = _scene_from_golden(g)
    bvh = GpuDynBVH()
    bvh.setGroup(golden_mesh(g))
    bvh.importTree(golden_tree(g))
    sc.spp, sc.seed = 1, 0
    out = bvh.render_frame(sc, sc.mesh.materials)
    ref = bvh.render_whitted(sc)
    assert out["shadow_rays"] == ref["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(g["img_rgb"]))


def test_flat_frame_spp16_matches_restatement(restatement):
    from conftest import golden_mesh, golden_tree, load_golden
    from test_gpu_render import _scene_from_golden
    from rfmanta_b200.dynbvh import GpuDynBVH
    for kind, name in ((0, "wald"), (1, "ks")):
        g = load_golden(name)
        sc = _scene_from_golden(g)
        sc.spp, sc.seed = 16, 99
        bvh = GpuDynBVH(tri_kind=kind)
        bvh.setGroup(golden_mesh(g))
        bvh.importTree(golden_tree(g))
        W = restatement.world(golden_tree(g), golden_mesh(g), tri_kind=kind)
        # all Lambertian, then material 0 a Phong (specular 0.5, exponent 20)
        for specpow in (None, np.array([20] + [-1] * (len(sc.mesh.materials) - 1), np.int32)):
            sc.specpow = specpow
            sc.specular = None if specpow is None else np.full(
                (len(sc.mesh.materials), 3), 0.5, np.float32)
            out = bvh.render_frame(sc, sc.mesh.materials)
            exp = restatement.render_frame(W, sc, sc.mesh.materials, specular=sc.specular,
                                           specpow=sc.specpow)
            assert out["shadow_rays"] == exp["shadow_rays"]
            assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))


def test_flat_scene_reports_no_instance():
    import torch
    from conftest import golden_mesh, golden_tree, load_golden
    from rfmanta_b200.dynbvh import GpuDynBVH
    g = load_golden("wald")
    bvh = GpuDynBVH()
    bvh.setGroup(golden_mesh(g))
    bvh.importTree(golden_tree(g))
    got = _trace(bvh, g["rand_org"], g["rand_dir"],
                 np.full(g["rand_org"].shape[1], 1e19, np.float32), False)
    assert np.all(got["inst"] == -1)
    assert np.array_equal(got["prim"], g["rand_prim"])
    torch.cuda.synchronize()


def test_instanced_scene_rejected_where_unsupported():
    from rfmanta_b200._lib import RQError
    from test_gpu_render import _scene_from_golden
    from conftest import load_golden
    g = load_instanced()
    top, inner = _device_scene(g)
    sc = _scene_from_golden(load_golden("wald"))
    with pytest.raises(RQError):
        top.render_whitted(sc)
    with pytest.raises(RQError):
        top.setGroup(sc.mesh)


def test_bad_instance_arguments():
    from rfmanta_b200.dynbvh import InstancedBVH
    from rfmanta_b200._lib import RQError
    g = load_instanced()
    top, inner = _device_scene(g)
    with pytest.raises(RQError):  # missing inner scene
        InstancedBVH(inner, np.array([0, 5], np.int32), np.zeros((2, 3), np.float32)).rebuild()
    with pytest.raises(RQError):  # a nested instance cannot move
        InstancedBVH(inner, np.array([0], np.int32), np.ones((1, 3), np.float32),
                     np.array([1], np.int32)).rebuild()
    with pytest.raises(RQError):  # unknown kind
        InstancedBVH(inner, np.array([0], np.int32), np.zeros((1, 3), np.float32),
                     np.array([7], np.int32)).rebuild()


def test_two_level_scene_refuses_updated_inner_scenes():
    """Instance boxes and inner descriptors are taken when the two-level
    scene is made; after an inner scene's mesh moves the two-level scene
    refuses to trace until it is made again."""
    from rfmanta_b200._lib import RQ_ERR_STATE, RQError
    from rfmanta_b200.dynbvh import InstancedBVH, RayBatch
    g = load_instanced()
    top, inner = _device_scene(g, import_trees=False)
    rays = RayBatch(g["rand_org"], g["rand_dir"])
    top.intersect(rays)
    m = inner[0].getGroup()
    m.vertices = (m.vertices * np.float32(1.01)).astype(np.float32)
    inner[0].update()
    with pytest.raises(RQError) as e:
        top.intersect(RayBatch(g["rand_org"], g["rand_dir"]))
    assert e.value.code == RQ_ERR_STATE
    again = InstancedBVH(inner, g["inst_scene"], g["translation"], g["kind"])
    again.rebuild()
    again.intersect(RayBatch(g["rand_org"], g["rand_dir"]))


def _pixels_from_samples(sample_rgb, spp):
    r = sample_rgb.reshape(-1, spp, 3)
    acc = np.zeros((r.shape[0], 3), np.float32)
    for s in range(spp):
        acc = (acc + r[:, s]).astype(np.float32)
    return (acc * np.float32(np.float32(1.0) / np.float32(spp))).astype(np.float32)


def test_reflective_phong_matches_reference_fixture():
    """Reflective Phong frames (Phong.cc:438-540 recursion) against the
    reference's samples: a flat scene whose materials reflect each other
    and the two-level scene with reflective InstanceT spheres."""
    import os
    import sys
    from conftest import GOLDEN
    sys.path.insert(0, GOLDEN)
    from make_golden import REFLECT
    from test_oracle_reflect import flat_case, load_reflect
    from rfmanta_b200.dynbvh import GpuDynBVH
    r = load_reflect()
    tree, mesh, sc, spec, specpow, refl = flat_case(r)
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.importTree(tree)
    sc.specular, sc.specpow, sc.reflectivity = spec, specpow, refl
    out = bvh.render_frame(sc, mesh.materials)
    assert out["shadow_rays"] == int(r["flat_shadow_rays"])
    exp = _pixels_from_samples(r["flat_sample_rgb"], sc.spp)
    assert np.array_equal(_bits(out["rgb"]), _bits(exp))
    g = load_instanced()
    top, inner = _device_scene(g)
    sc = tiny_scene_from_golden(g)
    sc.reflectivity = np.where(g["specpow"] >= 0, np.float32(REFLECT["instanced_refl"]),
                               np.float32(0)).astype(np.float32)
    out = top.render_frame(sc, g["materials"])
    assert out["shadow_rays"] == int(r["inst_shadow_rays"])
    assert np.array_equal(_bits(out["rgb"]), _bits(_pixels_from_samples(r["inst_sample_rgb"],
                                                                         sc.spp)))


@pytest.mark.parametrize("max_depth,cutoff", [(15, 0.01), (3, 0.01), (15, 0.3), (0, 0.01)])
def test_reflective_phong_gpu_built_matches_restatement(restatement, max_depth, cutoff):
    from oracle.pyoracle import Tree
    from rfmanta_b200.dynbvh import GpuDynBVH
    from rfmanta_b200.treeio import parse_dynbvh_blob
    from test_oracle_reflect import flat_case, load_reflect
    r = load_reflect()
    _, mesh, sc, spec, specpow, refl = flat_case(r)
    bvh = GpuDynBVH(tri_kind=1)
    bvh.setGroup(mesh)
    bvh.rebuild()
    f = parse_dynbvh_blob(bvh.exportBlob(), mesh.n_tris)
    W = restatement.world(Tree(f.bounds, f.child, f.children, f.axis, f.left_cheaper, f.ids),
                          mesh, tri_kind=1)
    sc.specular, sc.specpow, sc.reflectivity = spec, specpow, refl
    sc.max_depth, sc.importance_cutoff = max_depth, cutoff
    out = bvh.render_frame(sc, mesh.materials)
    exp = restatement.render_frame(W, sc, mesh.materials, specular=spec, specpow=specpow,
                                   reflectivity=refl, max_depth=max_depth, cutoff=cutoff)
    assert out["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(exp["rgb"]))
