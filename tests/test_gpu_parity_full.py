"""Device parity at the benchmark sizes.

The other device tests pin the CUDA path bit for bit on fixtures and small
scenes; these run the benchmark workloads at their full size and compare
a seeded sample of every one with the CPU restatement on the same
(GPU-built, exported) trees:

  * batched queries: the benchmark's 64 batches over its 8 resident scenes
    (10,240 to 5,120,000 triangles) plus one closest-hit and one any-hit
    batch of 20,000 rays per scene, all in one autotuned plan; every
    supplemental batch and a 2,000-ray sample of every benchmark batch are
    traced again by the restatement (t, triangle id, hit flag);
  * the coherent frame: 1920x1080, 4 spp over the 1024x1024 heightfield
    (nested DynBVH) and 64 InstanceT spheres; seven rows (13,440 pixels,
    53,760 samples) rendered by the restatement;
  * the path-traced frame: 1280x720, 16 spp, depth 4, 1,212,416
    triangles; six rows (7,680 pixels, 122,880 paths) traced by the
    restatement, pixel means compared bit for bit.

The maximum per-channel image error against the restatement is asserted
to be 0 (bit-exact) in both frames.  The restatement itself is pinned to
the reference (tests/test_oracle_*.py, including the full-size coherent
rows in tests/test_oracle_full_size.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _tree_of(bvh, n_objects=None):
    from oracle.pyoracle import Tree
    from rfmanta_b200.treeio import parse_dynbvh_blob
    t = parse_dynbvh_blob(bvh.exportBlob(), n_objects)
    return Tree(t.bounds, t.child, t.children, t.axis, t.left_cheaper, t.ids)


def test_batched_queries_full_size(restatement):
    import torch
    from rfmanta_b200 import scenes
    from rfmanta_b200.batch import BatchedQueries, QueryBatch
    from rfmanta_b200.dynbvh import GpuDynBVH
    meshes = [scenes.query_scene(i) for i in range(8)]
    bvhs = []
    for m in meshes:
        b = GpuDynBVH()
        b.setGroup(m)
        b.rebuild()
        bvhs.append(b)
    specs = scenes.query_batches()
    batches, host = [], []
    for k, (si, n, anyhit) in enumerate(specs):
        lo, hi = meshes[si].bounds()
        o, d, tm = scenes.query_rays_torch(n, lo, hi, anyhit, seed=1000 + k, device="cuda")
        batches.append(QueryBatch(si, o, d, tm, anyhit))
        host.append(None)
    extra0 = len(batches)
    for si, m in enumerate(meshes):
        lo, hi = m.bounds()
        for anyhit in (False, True):
            o, d, tm = scenes.query_rays_torch(20000, lo, hi, anyhit, seed=5000 + 2 * si + anyhit,
                                               device="cuda")
            batches.append(QueryBatch(si, o, d, tm, anyhit))
    bq = BatchedQueries(bvhs, batches)
    bq.autotune(reps=1)
    bq.launch()
    torch.cuda.synchronize()
    trees = [_tree_of(b) for b in bvhs]
    rng = np.random.default_rng(77)
    checked = np.zeros((8, 2), np.int64)
    for i, b in enumerate(batches):
        n = int(b.tmax.shape[0])
        sel = np.arange(n) if i >= extra0 else np.sort(rng.choice(n, min(n, 2000), replace=False))
        idx = torch.from_numpy(sel).cuda()
        o = b.org[:, idx].cpu().numpy()
        d = b.dir[:, idx].cpu().numpy()
        tm = b.tmax[idx].cpu().numpy()
        exp = restatement.trace(trees[b.scene], meshes[b.scene], o, d, tm, anyhit=b.anyhit)
        prim = bq.prim[i][idx].cpu().numpy()
        t = bq.t[i][idx].cpu().numpy()
        if b.anyhit:
            assert np.array_equal(prim >= 0, exp["hit"] > 0), i
        else:
            assert np.array_equal(prim, exp["prim"]), i
            assert np.array_equal(_bits(t), _bits(exp["t"])), i
        checked[b.scene, int(b.anyhit)] += len(sel)
    assert (checked >= 20000).all(), checked
    bq.close()


def test_coherent_frame_full_size_rows(restatement):
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH, InstancedBVH
    sc = scenes.coherent_scene()
    inner = []
    for m in sc.inner:
        b = GpuDynBVH()
        b.setGroup(m)
        b.rebuild()
        inner.append(b)
    top = InstancedBVH(inner, sc.inst_scene, sc.translation, sc.kind)
    top.rebuild()
    out = top.render_frame(sc, sc.materials)
    rgb = out["rgb"].reshape(sc.yres, sc.xres, 3)
    W = restatement.world(_tree_of(top, top.n_instances),
                          inner=[(_tree_of(b, m.n_tris), m) for b, m in zip(inner, sc.inner)],
                          inst_scene=sc.inst_scene, translation=sc.translation, kind=sc.kind)
    npx = 0
    for rows in ((0, 2), (359, 361), (540, 542), (1079, 1080)):
        exp = restatement.render_frame(W, sc, sc.materials, rows=rows, specular=sc.specular,
                                       specpow=sc.specpow)
        got = rgb[rows[0]:rows[1]].reshape(-1, 3)
        err = float(np.abs(got - exp["rgb"]).max())
        assert err == 0.0, f"rows {rows}: max per-channel error {err}"
        assert np.array_equal(_bits(got), _bits(exp["rgb"]))
        npx += got.shape[0]
    assert npx >= 10000
    assert np.count_nonzero(rgb) > 0


def test_path_frame_full_size_rows(restatement):
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.path_scene()
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    out = bvh.render_path(sc)
    rgb = out["rgb"].reshape(sc.yres, sc.xres, 3)
    tree = _tree_of(bvh)
    spp = sc.spp
    npx = 0
    for y0, y1 in ((0, 2), (360, 362), (718, 720)):
        p0, p1 = y0 * sc.xres * spp, y1 * sc.xres * spp
        exp = restatement.render_path(tree, sc, paths=(p0, p1))
        r = exp["rad"].reshape(-1, spp, 3)
        acc = np.zeros((r.shape[0], 3), np.float32)
        for s in range(spp):
            acc = (acc + r[:, s]).astype(np.float32)
        pix = (acc * np.float32(np.float32(1.0) / np.float32(spp))).astype(np.float32)
        got = rgb[y0:y1].reshape(-1, 3)
        err = float(np.abs(got - pix).max())
        assert err == 0.0, f"rows {y0}-{y1}: max per-channel error {err}"
        assert np.array_equal(_bits(got), _bits(pix))
        npx += got.shape[0]
    assert npx >= 7680
    assert np.count_nonzero(rgb) > 0
