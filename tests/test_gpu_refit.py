"""Refit of an animated mesh (rq_scene_update_vertices / GpuDynBVH.update)
against the reference's own refit: WaldTriangle::update + DynBVH::update
(Model/Groups/DynBVH.cc:1574-1581, 2012-2123) on the same moved vertices.
Tree bounds, queries and the shaded frame must agree bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _moved(v, k):
    """Seeded, non-rigid motion of the vertices (frame k of an animation)."""
    rng = np.random.default_rng(100 + k)
    w = np.sin(3.0 * v[:, [1, 2, 0]] + 0.7 * k).astype(np.float32)
    return (v + np.float32(0.04) * w + rng.normal(scale=0.002, size=v.shape)).astype(np.float32)


@pytest.mark.parametrize("tri_kind", [0, 1])
def test_refit_matches_reference(tri_kind, restatement):
    from oracle.pyoracle import Reference
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH, RayBatch
    from rfmanta_b200.treeio import parse_dynbvh_blob
    if not Reference.available():
        pytest.skip("reference library not built")
    sc = scenes.tiny_frame_scene()
    ref = Reference().scene(sc.mesh, tri_kind)
    bvh = GpuDynBVH(tri_kind=tri_kind)
    bvh.setGroup(sc.mesh)
    bvh.importTree(ref.tree())
    v0 = sc.mesh.vertices.copy()
    lo, hi = v0.min(0), v0.max(0)
    o, d, _, _ = scenes.random_rays(4096, lo - 0.3, hi + 0.3, seed=5)
    for k in range(1, 4):
        sc.mesh.vertices = _moved(v0, k)
        ref.update_vertices(sc.mesh.vertices)
        bvh.update()
        rt = ref.tree()
        f = parse_dynbvh_blob(bvh.exportBlob(), sc.mesh.n_tris)
        used = rt.bounds.shape[0]
        assert np.array_equal(_bits(f.bounds[:used]), _bits(rt.bounds)), "refitted boxes differ"
        assert np.array_equal(f.axis[:used], rt.axis)
        exp = ref.intersect(o, d, np.full(o.shape[1], 1e19, np.float32))
        rays = RayBatch(o, d)
        bvh.intersect(rays)
        assert np.array_equal(rays.hitPrim, exp["prim"])
        assert np.array_equal(_bits(rays.minT), _bits(exp["t"]))
        hit = exp["hit"] == 1
        assert np.array_equal(_bits(rays.u)[hit], _bits(exp["u"])[hit])
        img = bvh.render_whitted(sc)
        rimg = ref.render(sc)
        assert img["shadow_rays"] == rimg["shadow_rays"]
        assert np.array_equal(_bits(img["rgb"]), _bits(rimg["rgb"]))
        assert np.isclose(bvh.sahCost(), ref.sah_cost(), rtol=1e-6)
    ref.close()


def test_refit_gpu_built_tree_matches_restatement(restatement):
    """A GPU-built tree refitted to moved vertices: the exported tree
    replayed by the restatement gives the device's results."""
    from oracle.pyoracle import Tree
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    from rfmanta_b200.treeio import parse_dynbvh_blob
    sc = scenes.small_frame_scene(level=4, grid=30, xres=96, yres=80)
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    v0 = sc.mesh.vertices.copy()
    sc.mesh.vertices = _moved(v0, 2)
    bvh.update()
    f = parse_dynbvh_blob(bvh.exportBlob(), sc.mesh.n_tris)
    tree = Tree(f.bounds, f.child, f.children, f.axis, f.left_cheaper, f.ids)
    # every node box encloses its subtree's moved triangles
    img = bvh.render_whitted(sc)
    exp = restatement.render_whitted(tree, sc)
    assert img["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(_bits(img["rgb"]), _bits(exp["rgb"]))
    assert np.array_equal(img["prim"], exp["prim"])


def test_refit_rejects_bad_input():
    from rfmanta_b200 import scenes
    from rfmanta_b200._lib import RQError, check, lib
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.tiny_frame_scene()
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    v = np.zeros((sc.mesh.vertices.shape[0] + 1, 3), np.float32)
    with pytest.raises(RQError):
        check(lib.rq_scene_update_vertices(bvh.handle, v.ctypes.data, v.shape[0]))
