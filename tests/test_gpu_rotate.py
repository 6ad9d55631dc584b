"""The rotating update on the device (rq_scene_update_vertices_ex with
RQ_UPDATE_ROTATE, GpuDynBVH.update()): DynBVH::update as the reference
ships it (TREE_ROT 1: refit, leaf re-splits, tree rotations).

Checked bit for bit, frame after frame:
  * against the reference's own updated trees (tests/golden/tree_update.npz):
    every node field, object_ids, the per-node costs and nextFree;
  * against the CPU restatement (oracle/rq_oracle_update.c) on GPU-built
    trees, and on a sequence mixing rotating and topology-keeping updates;
  * queries and the shaded frame on the updated tree against the
    restatement replaying the reference's tree;
  * the reference's own Raytracer rendering through the C++ drop-in after
    the mesh moved, against the reference's DynBVH after the same update.
"""
import os

import numpy as np
import pytest

from oracle.pyoracle import DROPIN_SO
from test_oracle_update import FIELDS, _load, _state

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _device_state(bvh, n_tris):
    """The device tree as the restatement's DynTree (fields, costs, nextFree)."""
    from oracle.pyoracle import DynTree, Tree
    from rfmanta_b200.treeio import parse_dynbvh_blob
    f = parse_dynbvh_blob(bvh.exportBlob(), n_tris)
    costs, nf = bvh.update_state()
    t = Tree(f.bounds, f.child, f.children, f.axis, f.left_cheaper, f.ids)
    assert f.children.shape[0] == nf
    return DynTree(t, n_tris, costs=costs, next_free=nf)


def _same(got, exp, what):
    assert got.next_free == exp.next_free, (what, got.next_free, exp.next_free)
    n = exp.next_free
    for f in FIELDS:
        a, b = getattr(got, f), getattr(exp, f)
        if f != "ids":
            a, b = a[:n], b[:n]
        a = np.ascontiguousarray(a)
        b = np.ascontiguousarray(b)
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"{what}: {f} differs"


def _mesh(g, name, k):
    from rfmanta_b200.scenes import Mesh
    v = g[f"{name}_vertices{k}"] if k else g[f"{name}_vertices0"]
    ix = g[f"{name}_indices"]
    return Mesh(np.ascontiguousarray(v), ix, np.zeros(ix.shape[0], np.uint32),
                np.full((1, 3), 0.6, np.float32))


@pytest.mark.parametrize("tri_kind", [0, 1])
def test_matches_reference_fixture(tri_kind):
    from rfmanta_b200.dynbvh import GpuDynBVH
    g = _load()
    for name in (str(x) for x in g["names"]):
        mesh = _mesh(g, name, 0)
        bvh = GpuDynBVH(tri_kind=tri_kind)
        bvh.setGroup(mesh)
        bvh.importTree(_state(g, name, 0).tree())
        for k in range(1, 5):
            mesh.vertices = g[f"{name}_vertices{k}"]
            bvh.update()
            _same(_device_state(bvh, mesh.n_tris), _state(g, name, k), f"{name} frame {k}")


def test_queries_after_update_match_reference_tree(restatement):
    """Closest and any-hit queries on the device's updated tree equal the
    restatement replaying the reference's updated tree (t, id, u, v)."""
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH, RayBatch
    g = _load()
    name = "small"
    mesh = _mesh(g, name, 0)
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.importTree(_state(g, name, 0).tree())
    for k in range(1, 5):
        mesh.vertices = g[f"{name}_vertices{k}"]
        bvh.update()
        lo, hi = mesh.vertices.min(0), mesh.vertices.max(0)
        ref_tree = _state(g, name, k).tree()
        for anyhit, seed in ((False, 30 + k), (True, 40 + k)):
            o, d, tm, _ = scenes.random_rays(4096, lo - 0.3, hi + 0.3, seed=seed,
                                             anyhit_fraction=float(anyhit))
            if not anyhit:
                tm = np.full(o.shape[1], 1e19, np.float32)
            exp = restatement.trace(ref_tree, mesh, o, d, tm, anyhit=anyhit)
            r = RayBatch(o, d, tm, flags=RayBatch.AnyHit if anyhit else 0)
            bvh.intersect(r)
            assert np.array_equal(r.wasHit(), exp["hit"] > 0)
            if not anyhit:
                assert np.array_equal(r.hitPrim, exp["prim"])
                assert np.array_equal(_bits(r.minT), _bits(exp["t"]))
                h = exp["hit"] > 0
                assert np.array_equal(_bits(r.u[h]), _bits(exp["u"][h]))
                assert np.array_equal(_bits(r.v[h]), _bits(exp["v"][h]))


def test_frame_after_update_matches_restatement(restatement):
    from oracle.pyoracle import Tree
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    from rfmanta_b200.treeio import parse_dynbvh_blob
    sc = scenes.tiny_frame_scene()
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    v0 = sc.mesh.vertices.copy()
    for k in (1, 2):
        sc.mesh.vertices = scenes.animated_vertices(v0, k)
        bvh.update()
        f = parse_dynbvh_blob(bvh.exportBlob(), sc.mesh.n_tris)
        tree = Tree(f.bounds, f.child, f.children, f.axis, f.left_cheaper, f.ids)
        img = bvh.render_whitted(sc)
        exp = restatement.render_whitted(tree, sc)
        assert img["shadow_rays"] == exp["shadow_rays"]
        assert np.array_equal(img["prim"], exp["prim"])
        assert np.array_equal(_bits(img["rgb"]), _bits(exp["rgb"]))


def test_gpu_built_tree_matches_restatement(restatement):
    """A GPU-built tree (its own node numbering) updated over frames, with
    topology-keeping refits in between: device and restatement agree."""
    from oracle.pyoracle import DynTree, Tree
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    from rfmanta_b200.treeio import parse_dynbvh_blob
    sc = scenes.small_frame_scene(level=4, grid=30, xres=8, yres=8)
    mesh = sc.mesh
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.rebuild()
    f = parse_dynbvh_blob(bvh.exportBlob(), mesh.n_tris)
    mine = DynTree(Tree(f.bounds, f.child, f.children, f.axis, f.left_cheaper, f.ids),
                   mesh.n_tris, next_free=f.children.shape[0])
    restatement.tree_costs(mine)
    v0 = mesh.vertices.copy()
    for k, rotate in ((1, True), (2, False), (3, True), (4, True), (5, False), (6, True)):
        v = scenes.animated_vertices(v0, k, amplitude=0.03, seed=9)
        mesh.vertices = v
        bvh.update(rotate=rotate)
        restatement.tree_update(mine, v, mesh.indices, rotate=rotate)
        got = _device_state(bvh, mesh.n_tris)
        _same(got, mine, f"frame {k} rotate={rotate}")


def test_single_leaf_tree():
    """A tree that is one leaf: the update is its box (no rotation)."""
    from oracle.pyoracle import Tree
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH, RayBatch
    from rfmanta_b200.treeio import parse_dynbvh_blob
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], np.float32)
    ix = np.array([[0, 1, 2], [0, 2, 3], [1, 3, 4]], np.uint32)
    mesh = scenes.Mesh(v, ix, np.zeros(3, np.uint32), np.ones((1, 3), np.float32))
    b = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)[None]
    leaf = Tree(b, np.zeros(1, np.int32), np.array([3], np.int32), np.zeros(1, np.uint8),
                np.zeros(1, np.uint8), np.arange(3, dtype=np.int32))
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.importTree(leaf)
    mesh.vertices = v * np.float32(2.0)
    bvh.update()
    f = parse_dynbvh_blob(bvh.exportBlob(), 3)
    assert f.children[0] == 3
    assert np.array_equal(f.bounds[0], np.concatenate([v.min(0), v.max(0)]) * 2)
    r = RayBatch(np.array([[0.2], [0.2], [-5.0]], np.float32),
                 np.array([[0.0], [0.0], [1.0]], np.float32))
    bvh.intersect(r)
    assert r.hitPrim[0] == 0


def test_rejects_partial_trees():
    """The rotating update needs every triangle in exactly one leaf."""
    from oracle.pyoracle import Tree
    from rfmanta_b200 import scenes
    from rfmanta_b200._lib import RQ_ERR_STATE, RQError
    from rfmanta_b200.dynbvh import GpuDynBVH
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    ix = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    mesh = scenes.Mesh(v, ix, np.zeros(2, np.uint32), np.ones((1, 3), np.float32))
    b = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)[None]
    leaf = Tree(b, np.zeros(1, np.int32), np.array([1], np.int32), np.zeros(1, np.uint8),
                np.zeros(1, np.uint8), np.array([0, 1], np.int32))
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.importTree(leaf)
    with pytest.raises(RQError) as e:
        bvh.update()
    assert e.value.code == RQ_ERR_STATE
    bvh.update(rotate=False)  # the topology-keeping refit still works


@pytest.mark.skipif(not os.path.exists(DROPIN_SO), reason="oracle/_ref/libmanta_dropin.so not built")
def test_dropin_renders_after_update(tmp_path):
    """Manta's Raytracer through GpuDynBVH after GpuDynBVH::update equals
    Manta's Raytracer through DynBVH after DynBVH::update."""
    from oracle.pyoracle import Reference
    from rfmanta_b200 import scenes
    sc = scenes.small_frame_scene(level=4, grid=30, xres=128, yres=128)
    ref = Reference(path=DROPIN_SO)
    cpu = ref.scene(sc.mesh, 0)
    gpu = ref.scene(sc.mesh, 0)
    gpu.use_gpu(0, 0, tree_file=str(tmp_path / "tree.bvh"))
    v0 = sc.mesh.vertices.copy()
    for k in (1, 2, 3):
        v = scenes.animated_vertices(v0, k, amplitude=0.03, seed=5)
        cpu.update_vertices(v)
        gpu.update_vertices(v)
        want = cpu.render(sc, nthreads=4)
        got = gpu.render(sc, nthreads=4)
        assert got["shadow_rays"] == want["shadow_rays"]
        assert np.array_equal(got["prim"], want["prim"])
        assert np.array_equal(_bits(got["rgb"]), _bits(want["rgb"]))


def test_update_from_device_vertices_equals_host_update():
    """rq_scene_update_vertices_device gives the tree the host-pointer call
    gives, and the scene's host copy of the vertices follows (it feeds the
    instance boxes of a two-level scene built on it)."""
    import torch
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH, InstancedBVH
    sc = scenes.tiny_frame_scene()
    v0 = sc.mesh.vertices.copy()
    from oracle.pyoracle import Tree
    from rfmanta_b200.treeio import parse_dynbvh_blob
    a, b = GpuDynBVH(), GpuDynBVH()
    a.setGroup(sc.mesh)
    a.rebuild()
    f0 = parse_dynbvh_blob(a.exportBlob(), sc.mesh.n_tris)
    b.setGroup(sc.mesh)
    b.importTree(Tree(f0.bounds, f0.child, f0.children, f0.axis, f0.left_cheaper, f0.ids))
    for k in (1, 2, 3):
        v = scenes.animated_vertices(v0, k)
        sc.mesh.vertices = v
        a.update(rotate=k != 2)
        dv = torch.from_numpy(v).cuda()
        b.update_device(dv.data_ptr(), rotate=k != 2)
        torch.cuda.synchronize()
        assert a.exportBlob() == b.exportBlob()
    top = InstancedBVH([b], np.array([0], np.int32), np.zeros((1, 3), np.float32))
    top.rebuild()
    t = parse_dynbvh_blob(top.exportBlob(), 1)
    assert np.array_equal(t.bounds[0, :3], v.min(0)) and np.array_equal(t.bounds[0, 3:], v.max(0))
