"""Refit of an animated mesh (rq_scene_update_vertices / GpuDynBVH.update).

The device refit keeps the tree's topology and recomputes every box bottom
up (DynBVH::updateBounds, Model/Groups/DynBVH.cc:2064-2123).  The
reference's DynBVH::update additionally applies Kopta et al.'s tree
rotations and approximate leaf splits (TREE_ROT = 1, DynBVH.h:377,
rotateNode DynBVH.cc:3047-3330), so after an update the two trees differ in
shape.  Checked here:
  * every refitted box is the exact union of its children / triangles;
  * closest-hit and any-hit queries and the shaded frame on the refitted
    tree agree with the reference's own updated tree on every ray except
    near-ties (two candidate hits within 1e-6 relative in t, where the
    traversal order may pick either; found with the restatement's top-2
    pass);
  * a GPU-built tree refitted to moved vertices replays bit for bit in the
    restatement.
"""
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


def _check_boxes(f, mesh):
    """Node boxes = exact unions (leaf: its triangles' vertices)."""
    tri_lo = mesh.vertices[mesh.indices].min(axis=1)
    tri_hi = mesh.vertices[mesh.indices].max(axis=1)

    def box(n):
        if f.children[n] != 0:
            ids = f.ids[f.child[n]:f.child[n] + f.children[n]]
            return tri_lo[ids].min(0), tri_hi[ids].max(0)
        (l0, l1), (r0, r1) = box(f.child[n]), box(f.child[n] + 1)
        return np.minimum(l0, r0), np.maximum(l1, r1)

    def walk(n):
        lo, hi = box(n)
        assert np.array_equal(_bits(f.bounds[n, :3]), _bits(lo)), n
        assert np.array_equal(_bits(f.bounds[n, 3:]), _bits(hi)), n
        if f.children[n] == 0:
            walk(f.child[n])
            walk(f.child[n] + 1)
    walk(0)


@pytest.mark.parametrize("tri_kind", [0, 1])
def test_refit_matches_reference(tri_kind, restatement):
    import sys
    from oracle.pyoracle import Reference, Tree
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH, RayBatch
    from rfmanta_b200.treeio import parse_dynbvh_blob
    if not Reference.available():
        pytest.skip("reference library not built")
    sys.setrecursionlimit(10000)
    sc = scenes.tiny_frame_scene()
    ref = Reference().scene(sc.mesh, tri_kind)
    bvh = GpuDynBVH(tri_kind=tri_kind)
    bvh.setGroup(sc.mesh)
    bvh.importTree(ref.tree())
    v0 = sc.mesh.vertices.copy()
    lo, hi = v0.min(0), v0.max(0)
    o, d, _, _ = scenes.random_rays(4096, lo - 0.3, hi + 0.3, seed=5)
    oa, da, ta, _ = scenes.random_rays(4096, lo - 0.3, hi + 0.3, seed=6, anyhit_fraction=1.0)
    tmax = np.full(o.shape[1], 1e19, np.float32)
    for k in range(1, 4):
        sc.mesh.vertices = _moved(v0, k)
        ref.update_vertices(sc.mesh.vertices)
        bvh.update()
        f = parse_dynbvh_blob(bvh.exportBlob(), sc.mesh.n_tris)
        _check_boxes(f, sc.mesh)
        tree = Tree(f.bounds, f.child, f.children, f.axis, f.left_cheaper, f.ids)
        t1, t2, _, p2 = restatement.top2(tree, sc.mesh, o, d, tmax, tri_kind=tri_kind)
        tie = (p2 >= 0) & (np.abs(t2 - t1) <= 1e-6 * np.abs(t1))
        exp = ref.intersect(o, d, tmax)
        rays = RayBatch(o, d)
        bvh.intersect(rays)
        ok = ~tie
        assert np.count_nonzero(tie) < 0.01 * tie.size
        assert np.array_equal(rays.hitPrim[ok], exp["prim"][ok])
        assert np.array_equal(_bits(rays.minT[ok]), _bits(exp["t"][ok]))
        hit = ok & (exp["hit"] == 1)
        assert np.array_equal(_bits(rays.u[hit]), _bits(exp["u"][hit]))
        # occlusion does not depend on the tree's shape
        expa = ref.intersect(oa, da, ta, anyhit=True)
        ra = RayBatch(oa, da, ta, flags=RayBatch.AnyHit)
        bvh.intersect(ra)
        assert np.array_equal(ra.wasHit(), expa["hit"] > 0)
        img = bvh.render_whitted(sc)
        rimg = ref.render(sc)
        same = img["prim"] == rimg["prim"]
        assert np.count_nonzero(~same) <= np.count_nonzero(tie) + 2
        assert np.array_equal(_bits(img["rgb"][same]), _bits(rimg["rgb"][same]))
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
