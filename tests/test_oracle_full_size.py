"""The restatement against the live reference on the coherent frame at its
benchmark size: the 1024x1024 heightfield (2,097,152 triangles, nested
DynBVH) plus 64 InstanceT copies of a level-6 displaced icosphere, 1920x1080
at 4 spp.  The reference builds its own trees (DynBVH::rebuild) and renders
the samples of seven rows with Raytracer::traceEyeRays
(Engine/Renderers/Raytracer.cc:41-97) through InstanceT
(Model/Instances/InstanceT.cc:60-90); the restatement renders the same rows
over the reference's trees.  Per-sample colours and triangle ids must be
bit-identical; the device is tied to the restatement on the same rows in
tests/test_gpu_parity_full.py.  Needs the reference checker library
(oracle/_ref); skipped without it."""
import numpy as np
import pytest

ROWS = ((0, 2), (359, 361), (540, 542), (1079, 1080))


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_coherent_rows_full_size(restatement):
    from oracle.pyoracle import Reference
    from rfmanta_b200 import scenes
    if not Reference.available():
        pytest.skip("reference library not built")
    ref = Reference()
    sc = scenes.coherent_scene()
    inner = [ref.scene(m, 0) for m in sc.inner]
    for r in inner:
        for m, sp in enumerate(sc.specpow):
            if sp >= 0:
                r.set_phong(m, sc.specular[m], int(sp))
    top = ref.instanced(inner, sc.inst_scene, sc.translation, sc.kind)
    W = restatement.world(top.tree(), inner=[(r.tree(), m) for r, m in zip(inner, sc.inner)],
                          inst_scene=sc.inst_scene, translation=sc.translation, kind=sc.kind)
    npx = 0
    for y0, y1 in ROWS:
        i0, i1 = y0 * sc.xres * sc.spp, y1 * sc.xres * sc.spp
        px, py = restatement.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed, items=(i0, i1))
        img = top.render_coords(sc, px, py, nthreads=8)
        out = restatement.render_frame(W, sc, sc.materials, rows=(y0, y1), per_sample=True,
                                       specular=sc.specular, specpow=sc.specpow)
        assert np.array_equal(out["sample_prim"], img["prim"]), (y0, y1)
        err = float(np.abs(out["sample_rgb"] - img["rgb"]).max())
        assert err == 0.0, f"rows {y0}-{y1}: max per-channel error {err}"
        assert np.array_equal(_bits(out["sample_rgb"]), _bits(img["rgb"]))
        npx += (y1 - y0) * sc.xres
    assert npx >= 10000
    top.close()
    for r in inner:
        r.close()
