"""The animated-mesh update on the CPU: the restatement
(oracle/rq_oracle_update.c) of DynBVH::update (Model/Groups/DynBVH.cc:
1574-1581, 2012-2123) with its tree rotations and leaf re-splits
(rotateNode 3051-3348, TREE_ROT 1 in DynBVH.h:377) against the reference.

Pinned by the committed fixture tests/golden/tree_update.npz (the
reference's tree, per-node costs and nextFree after each of four frames) and,
where the reference library is built, live on a larger mesh.  Every field
must agree bit for bit: the node boxes, child/children, split axes,
isLeftCheaper, the costs the next frame's rotations start from, object_ids
and nextFree."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

FIELDS = ("bounds", "child", "children", "axis", "left_cheaper", "costs", "ids")


def _load():
    z = np.load(os.path.join(GOLDEN, "tree_update.npz"))
    return {k: z[k] for k in z.files}


def _state(g, name, k):
    from oracle.pyoracle import DynTree, Tree
    p = f"{name}_s{k}_"
    t = Tree(g[p + "bounds"], g[p + "child"], g[p + "children"], g[p + "axis"],
             g[p + "left_cheaper"], g[p + "ids"])
    return DynTree(t, g[p + "ids"].shape[0], costs=g[p + "costs"],
                   next_free=int(g[p + "next_free"]), cap=int(g[p + "cap"]))


def assert_same_state(got, exp, what=""):
    assert got.next_free == exp.next_free, (what, got.next_free, exp.next_free)
    n = exp.next_free
    for f in FIELDS:
        a, b = getattr(got, f), getattr(exp, f)
        if f != "ids":
            a, b = a[:n], b[:n]
        a = np.ascontiguousarray(a)
        b = np.ascontiguousarray(b)
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"{what}: {f} differs"


def test_fixture_frames(restatement):
    from oracle.pyoracle import Tree
    g = _load()
    for name in (str(x) for x in g["names"]):
        t = _state(g, name, 0)
        # a rebuild leaves computeCost<true> in the costs
        exp_costs = t.costs.copy()
        t.costs[:] = 0
        restatement.tree_costs(t)
        assert np.array_equal(t.costs.view(np.uint32), exp_costs.view(np.uint32))
        s0 = _state(g, name, 0)
        for k in range(1, 5):
            restatement.tree_update(t, g[f"{name}_vertices{k}"], g[f"{name}_indices"])
            exp = _state(g, name, k)
            assert_same_state(t, exp, f"{name} frame {k}")
        # the fixture exercises both halves of rotateNode
        assert t.next_free > s0.next_free, "no leaf was re-split"
        assert np.count_nonzero(t.child[:s0.next_free] != s0.child[:s0.next_free]) > 10
        assert isinstance(t.tree(), Tree)


def test_refit_only_mode_keeps_topology(restatement):
    """rotate=0 restates the reference built with TREE_ROT 0: boxes only."""
    g = _load()
    t = _state(g, "small", 0)
    s0 = _state(g, "small", 0)
    v = g["small_vertices2"]
    ix = g["small_indices"]
    restatement.tree_update(t, v, ix, rotate=False)
    n = s0.next_free
    assert t.next_free == n
    for f in ("child", "children", "left_cheaper", "ids", "costs"):
        assert np.array_equal(getattr(t, f)[:n], getattr(s0, f)[:n]), f
    tri = v[ix.astype(np.int64)]
    lo, hi = tri.min(axis=1), tri.max(axis=1)
    for i in range(n):
        if t.children[i] != 0:
            ids = t.ids[t.child[i]:t.child[i] + t.children[i]]
            assert np.array_equal(t.bounds[i, :3], lo[ids].min(0))
            assert np.array_equal(t.bounds[i, 3:], hi[ids].max(0))
            assert t.axis[i] == 0


def test_live_reference_larger_mesh(restatement):
    from oracle.pyoracle import DynTree, Reference
    from rfmanta_b200 import scenes
    if not Reference.available():
        pytest.skip("reference library not built")
    ref = Reference()
    mesh = scenes.small_frame_scene(level=4, grid=30, xres=8, yres=8).mesh
    rs = ref.scene(mesh, 0)
    d0 = rs.dyn_tree()
    mine = DynTree(rs.tree(), mesh.n_tris, next_free=d0.next_free, cap=d0.cap)
    restatement.tree_costs(mine)
    assert np.array_equal(mine.costs[:d0.next_free].view(np.uint32),
                          d0.costs[:d0.next_free].view(np.uint32))
    v0 = mesh.vertices.copy()
    for k in (1, 2, 3):
        v = scenes.animated_vertices(v0, k, amplitude=0.03, seed=7)
        rs.update_vertices(v)
        restatement.tree_update(mine, v, mesh.indices)
        assert_same_state(mine, rs.dyn_tree(), f"frame {k}")
    rs.close()
