"""The path tracer's estimator against the reference's, in expectation.

The reference's KajiyaPathtracer draws its random numbers per packet and
thread, so no path of it can be replayed one for one; the device path
tracer is pinned bit for bit to the CPU restatement instead
(tests/test_gpu_path.py), and the restatement is pinned here to the
reference's images: 16 independent renders of each at 4096 samples per
pixel (the reference's in tests/golden/path_stats.npz, made by
tests/golden/make_golden.py with one thread so each seed is reproducible)
must agree in every pixel's mean and in the image mean within their
sampling error.  This is what catches a difference in the light transport:
the reference's Russian roulette leaves survivors unscaled
(KajiyaPathtracer.cc:468-475 rescales the rays it just killed), which
darkens its images by 0.1% here; a 1/p-weighted roulette is 10 standard
errors away.
"""
import os

import numpy as np

from conftest import GOLDEN


def _ours(restatement, tree, sc, seeds):
    out = []
    for s in seeds:
        sc.seed = int(s)
        out.append(restatement.render_path(tree, sc)["rgb"].reshape(sc.yres, sc.xres, 3))
    return np.array(out, np.float64)


def _z(a, b):
    """Welch z of the means over the first axis."""
    va = a.var(0, ddof=1) / a.shape[0]
    vb = b.var(0, ddof=1) / b.shape[0]
    return (a.mean(0) - b.mean(0)) / np.sqrt(va + vb + 1e-30)


import pytest


@pytest.mark.parametrize("with_ambient", [False, True])
def test_images_match_reference_in_expectation(restatement, with_ambient):
    """At depth 4, and at depth 2 with a ConstantAmbient light (added where
    a path reaches its last bounce, do_ambient_on_maxdepth)."""
    from oracle.pyoracle import Tree
    from rfmanta_b200 import scenes
    z = np.load(os.path.join(GOLDEN, "path_stats.npz"))
    ref = z["images_ambient" if with_ambient else "images"].astype(np.float64)
    xres, yres, spp = int(z["xres"]), int(z["yres"]), int(z["spp"])
    sc = scenes.tiny_path_scene(xres=xres, yres=yres, spp=spp)
    if with_ambient:  # depth 2: most paths reach the last bounce
        sc.ambient, sc.max_depth = tuple(float(x) for x in z["ambient"]), 2
    assert ref.shape[1:] == (yres, xres, 3)
    # the image's expectation does not depend on the tree, so any valid tree
    # over the mesh serves (a median split, built here without a GPU)
    tree = _median_tree(sc.mesh)
    assert isinstance(tree, Tree)
    ours = _ours(restatement, tree, sc, range(3000, 3000 + ref.shape[0]))
    img_z = _z(ours.mean((1, 2)), ref.mean((1, 2)))
    assert np.all(np.abs(img_z) < 4.0), img_z
    pix_z = _z(ours, ref)
    assert abs(pix_z.mean()) < 0.3, pix_z.mean()
    assert np.mean(np.abs(pix_z) > 4.0) < 0.01
    # the check has the power to see a 0.1% bias
    biased = _z((ours * 1.001).mean((1, 2)), ref.mean((1, 2)))
    assert np.all(np.abs(biased) > 4.0), biased
    if with_ambient:  # and the ambient term is there to be seen
        sc.ambient = (0.0, 0.0, 0.0)
        dark = _ours(restatement, tree, sc, range(4000, 4008))
        assert np.all(np.abs(_z(dark.mean((1, 2)), ref.mean((1, 2)))) > 8.0)


def _median_tree(mesh):
    """A valid DynBVH tree over the mesh: median splits on the longest
    centroid axis, leaves of up to 4 triangles (node boxes exact)."""
    from oracle.pyoracle import Tree
    tri = mesh.vertices[mesh.indices.astype(np.int64)]
    lo, hi = tri.min(1), tri.max(1)
    cen = 0.5 * (lo + hi)
    bounds, child, children, axis = [None], [0], [0], [0]
    ids = []

    def build(node, objs):
        b = np.concatenate([lo[objs].min(0), hi[objs].max(0)]).astype(np.float32)
        bounds[node] = b
        if len(objs) <= 4:
            child[node] = len(ids)
            children[node] = len(objs)
            ids.extend(sorted(int(o) for o in objs))
            return
        ax = int(np.argmax(cen[objs].max(0) - cen[objs].min(0)))
        order = objs[np.argsort(cen[objs, ax], kind="stable")]
        half = len(order) // 2
        c = len(bounds)
        bounds.extend([None, None])
        child.extend([0, 0])
        children.extend([0, 0])
        axis.extend([0, 0])
        child[node] = c
        children[node] = 0
        axis[node] = ax
        build(c, order[:half])
        build(c + 1, order[half:])

    build(0, np.arange(mesh.n_tris))
    n = len(bounds)
    return Tree(np.array(bounds, np.float32), np.array(child, np.int32),
                np.array(children, np.int32), np.array(axis, np.uint8),
                np.zeros(n, np.uint8), np.array(ids, np.int32))
