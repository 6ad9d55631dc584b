"""Reflective Phong on the CPU: the restatement's recursion (oracle/
rq_oracle.c trace_color) against the reference's Phong::shade reflection
(Model/Materials/Phong.cc:438-540) and Raytracer recursion, bit for bit per
image sample, with the reference's default RenderParameters (maxDepth 15,
importance cutoff 0.01).  Pinned by tests/golden/tiny_reflect.npz (a flat
scene whose two materials reflect each other, and the tiny two-level scene
with reflective InstanceT spheres) and live where the reference is built.

The reference extends a run of reflected rays to the end of its packet once
the run's first ray passes the importance cutoff (its while loop re-tests
that first ray); per-ray cutoffs agree with it wherever the rays of a packet
carry the same importance, as they do here (one reflective material, or
importances that stay above the cutoff)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from test_oracle_instance import golden_world, load_instanced, tiny_scene_from_golden


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def load_reflect():
    z = np.load(os.path.join(GOLDEN, "tiny_reflect.npz"))
    return {k: z[k] for k in z.files}


def flat_case(g):
    """(tree, mesh, scene, specular, specpow, reflectivity) of the flat case."""
    from make_golden import REFLECT
    from oracle.pyoracle import Tree
    from rfmanta_b200 import scenes
    tree = Tree(*[g[f"flat_{f}"] for f in ("bounds", "child", "children", "axis",
                                          "left_cheaper", "ids")])
    mesh = scenes.Mesh(g["flat_vertices"], g["flat_indices"], g["flat_face_material"],
                       g["flat_materials"])
    sc = scenes.tiny_frame_scene(xres=40, yres=32)
    sc.mesh = mesh
    sc.spp, sc.seed = 4, 5
    n = mesh.materials.shape[0]
    spec = np.full((n, 3), 0.4, np.float32)
    specpow = np.array(REFLECT["flat_specpow"][:n], np.int32)
    refl = np.array(REFLECT["flat_refl"][:n], np.float32)
    return tree, mesh, sc, spec, specpow, refl


def _golden_dir():
    import sys
    d = os.path.join(GOLDEN)
    if d not in sys.path:
        sys.path.insert(0, d)


def test_flat_fixture(restatement):
    _golden_dir()
    g = load_reflect()
    tree, mesh, sc, spec, specpow, refl = flat_case(g)
    W = restatement.world(tree, mesh)
    out = restatement.render_frame(W, sc, mesh.materials, per_sample=True, specular=spec,
                                   specpow=specpow, reflectivity=refl)
    assert out["shadow_rays"] == int(g["flat_shadow_rays"])
    assert np.array_equal(out["sample_prim"], g["flat_sample_prim"])
    assert np.array_equal(_bits(out["sample_rgb"]), _bits(g["flat_sample_rgb"]))
    # the reflections are there: without them the image differs
    plain = restatement.render_frame(W, sc, mesh.materials, per_sample=True, specular=spec,
                                     specpow=specpow)
    assert np.count_nonzero((plain["sample_rgb"] != out["sample_rgb"]).any(1)) > 100
    assert plain["shadow_rays"] < out["shadow_rays"]


def test_instanced_fixture(restatement):
    _golden_dir()
    from make_golden import REFLECT
    g = load_instanced()
    r = load_reflect()
    W = golden_world(restatement, g)
    sc = tiny_scene_from_golden(g)
    refl = np.where(g["specpow"] >= 0, np.float32(REFLECT["instanced_refl"]),
                    np.float32(0)).astype(np.float32)
    out = restatement.render_frame(W, sc, g["materials"], per_sample=True,
                                   specular=g["specular"], specpow=g["specpow"],
                                   reflectivity=refl)
    assert out["shadow_rays"] == int(r["inst_shadow_rays"])
    assert np.array_equal(out["sample_prim"], r["inst_sample_prim"])
    assert np.array_equal(_bits(out["sample_rgb"]), _bits(r["inst_sample_rgb"]))


def test_live_reference_depth_and_cutoff(restatement):
    """Other recursion limits, live: maxDepth 2 and a cutoff that stops the
    chain after two reflections (one reflective material)."""
    from oracle.pyoracle import Reference
    from rfmanta_b200 import scenes
    if not Reference.available():
        pytest.skip("reference library not built")
    ref = Reference()
    sc = scenes.tiny_frame_scene(xres=24, yres=20)
    sc.spp, sc.seed = 4, 9
    m = sc.mesh
    for max_depth, cutoff in ((2, 0.01), (15, 0.2)):
        rs = ref.scene(m, 0)
        rs.set_phong(0, np.full(3, 0.3, np.float32), 12, 0.5)
        rs.set_render_parameters(max_depth, cutoff)
        px, py = restatement.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed)
        img = rs.render_coords(sc, px, py)
        W = restatement.world(rs.tree(), m)
        n = m.materials.shape[0]
        specpow = np.full(n, -1, np.int32)
        specpow[0] = 12
        refl = np.zeros(n, np.float32)
        refl[0] = 0.5
        out = restatement.render_frame(W, sc, m.materials, per_sample=True,
                                       specular=np.full((n, 3), 0.3, np.float32),
                                       specpow=specpow, reflectivity=refl,
                                       max_depth=max_depth, cutoff=cutoff)
        assert out["shadow_rays"] == img["shadow_rays"], (max_depth, cutoff)
        assert np.array_equal(_bits(out["sample_rgb"]), _bits(img["rgb"])), (max_depth, cutoff)
        rs.close()
