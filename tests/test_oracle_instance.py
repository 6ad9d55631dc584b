"""Two-level scenes on the CPU: the restatement (oracle/rq_oracle.c world
traversal and supersampled frame) against the reference's own DynBVH over
InstanceT objects, bit for bit.

Pinned twice: against the committed fixture tests/golden/tiny_instanced.npz
(made by tests/golden/make_golden.py from the reference), and, where the
reference library is built, against the live reference on further cases
(Kensler-Shirley triangles, other seeds).  Reference-side notes, each tested
here:
  * InstanceT::intersect (Model/Instances/InstanceT.cc:60-90) reports the
    inner triangle through its MPT scratchpad and keeps the inner u/v in its
    own packet, so u/v are compared only for hits outside an InstanceT;
  * the spheres are Phong (Model/Materials/Phong.cc, scalar branch, no
    reflection), the heightfield Lambertian;
  * an AnyHit query never reports occlusion inside an InstanceT: the inner
    DynBVH pins minT to T_EPSILON (DynBVH.cc:331-349) and RayPacket::hit
    rejects t = T_EPSILON (RayPacket.h:531-543); a nested DynBVH object
    does occlude.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

KEYS = ("hit", "t", "prim")


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def load_instanced():
    z = np.load(os.path.join(GOLDEN, "tiny_instanced.npz"))
    return {k: z[k] for k in z.files}


def golden_world(rs, g, tri_kind=0):
    from oracle.pyoracle import Tree
    from rfmanta_b200.scenes import Mesh

    def tree(name):
        return Tree(*[g[f"{name}_{f}"] for f in ("bounds", "child", "children", "axis",
                                                 "left_cheaper", "ids")])
    inner = []
    for i in range(int(g["n_inner"])):
        m = Mesh(g[f"inner{i}_vertices"], g[f"inner{i}_indices"],
                 g[f"inner{i}_face_material"], g["materials"])
        inner.append((tree(f"inner{i}"), m))
    return rs.world(tree("top"), inner=inner, inst_scene=g["inst_scene"],
                    translation=g["translation"], kind=g["kind"], tri_kind=tri_kind)


def tiny_scene_from_golden(g):
    from rfmanta_b200 import scenes
    sc = scenes.tiny_coherent_scene()
    assert (sc.xres, sc.yres, sc.spp, sc.seed) == (int(g["xres"]), int(g["yres"]),
                                                   int(g["spp"]), int(g["seed"]))
    assert np.array_equal(sc.specpow, g["specpow"]) and np.array_equal(sc.specular, g["specular"])
    return sc


def compare_queries(got, exp, kind_of_inst):
    for k in KEYS:
        a, b = (_bits(got[k]), _bits(exp[k])) if k == "t" else (got[k], exp[k])
        assert np.array_equal(a, b), f"{k}: {np.count_nonzero(a != b)} rays differ"
    # u/v only where the reference keeps them (no InstanceT in between)
    outside = (exp["hit"] == 1) & (exp["inst"] < 0)
    for k in ("u", "v"):
        assert np.array_equal(_bits(got[k])[outside], _bits(exp[k])[outside])
    # the reference names the instance only for InstanceT hits
    ihit = exp["inst"] >= 0
    assert np.array_equal(got["inst"][ihit], exp["inst"][ihit])
    nested = (got["hit"] == 1) & (exp["inst"] < 0)
    assert np.all(kind_of_inst[got["inst"][nested]] == 1)


def test_fixture_queries(restatement):
    g = load_instanced()
    W = golden_world(restatement, g)
    for tag, anyhit in (("rand", False), ("any", True)):
        tmax = g["any_tmax"] if anyhit else np.full(g[f"{tag}_org"].shape[1], 1e19, np.float32)
        got = restatement.trace_world(W, g[f"{tag}_org"], g[f"{tag}_dir"], tmax, anyhit)
        exp = {k: g[f"{tag}_{k}"] for k in ("hit", "t", "prim", "u", "v", "inst")}
        if anyhit:
            # the query's own output t for occluded rays is T_EPSILON on both
            assert np.count_nonzero(exp["hit"]) > 100
        else:
            assert np.count_nonzero(exp["inst"] >= 0) > 50, "too few InstanceT hits"
        compare_queries(got, exp, g["kind"])


def test_fixture_frame_samples(restatement):
    g = load_instanced()
    W = golden_world(restatement, g)
    sc = tiny_scene_from_golden(g)
    px, py = restatement.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed)
    assert np.array_equal(_bits(px), _bits(g["sample_px"]))
    assert np.array_equal(_bits(py), _bits(g["sample_py"]))
    assert np.any(g["specpow"] >= 0), "the fixture has a Phong material"
    out = restatement.render_frame(W, sc, g["materials"], per_sample=True,
                                   specular=g["specular"], specpow=g["specpow"])
    assert out["shadow_rays"] == int(g["shadow_rays"])
    assert np.array_equal(out["sample_prim"], g["sample_prim"])
    assert np.array_equal(_bits(out["sample_t"]), _bits(g["sample_t"]))
    err = np.abs(out["sample_rgb"] - g["sample_rgb"]).max()
    assert err == 0.0, f"max per-channel error {err}"
    assert np.array_equal(_bits(out["sample_rgb"]), _bits(g["sample_rgb"]))
    # the pixel colour is the samples' sum in sample order times 1/spp
    r = g["sample_rgb"].reshape(-1, sc.spp, 3)
    acc = np.zeros((r.shape[0], 3), np.float32)
    for s in range(sc.spp):
        acc = (acc + r[:, s]).astype(np.float32)
    pix = (acc * np.float32(np.float32(1.0) / np.float32(sc.spp))).astype(np.float32)
    assert np.array_equal(_bits(out["rgb"]), _bits(pix))


def test_instances_cast_no_anyhit_occlusion_in_reference(restatement):
    """A shadow ray straight through an InstanceT sphere is not occluded,
    through the nested heightfield it is (reference fixture and restatement
    agree)."""
    g = load_instanced()
    W = golden_world(restatement, g)
    k = int(np.nonzero(g["kind"] == 0)[0][0])
    c = g["translation"][k]
    org = np.array([[c[0] + 0.3], [c[1] + 3.0], [c[2] + 0.2]], np.float32)
    d = np.array([-0.3, -3.0, -0.2])
    dir = (d / np.linalg.norm(d)).astype(np.float32).reshape(3, 1)
    closest = restatement.trace_world(W, org, dir, np.array([1e19], np.float32), False)
    assert closest["hit"][0] == 1 and closest["inst"][0] == k
    shadow = restatement.trace_world(W, org, dir, np.array([1e19], np.float32), True)
    assert shadow["hit"][0] == 1 and shadow["inst"][0] == 0  # the heightfield below
    short = np.array([np.float32(closest["t"][0]) + np.float32(0.1)], np.float32)
    shadow = restatement.trace_world(W, org, dir, short, True)
    assert shadow["hit"][0] == 0


def _live_reference():
    from oracle.pyoracle import Reference
    if not Reference.available():
        pytest.skip("reference library not built")
    return Reference()


@pytest.mark.parametrize("tri_kind", [0, 1])
def test_live_reference(restatement, tri_kind):
    from rfmanta_b200 import scenes
    ref = _live_reference()
    sc = scenes.coherent_scene(hf_n=10, n_instances=9, sphere_level=1, xres=32, yres=24,
                               spp=4, seed=41)
    inner = [ref.scene(m, tri_kind) for m in sc.inner]
    for r in inner:
        for m, sp in enumerate(sc.specpow):
            if sp >= 0:
                r.set_phong(m, sc.specular[m], int(sp))
    top = ref.instanced(inner, sc.inst_scene, sc.translation, sc.kind)
    W = restatement.world(top.tree(), inner=[(r.tree(), m) for r, m in zip(inner, sc.inner)],
                          inst_scene=sc.inst_scene, translation=sc.translation, kind=sc.kind,
                          tri_kind=tri_kind)
    lo = np.array([-4.5, -0.5, -4.5], np.float32)
    hi = np.array([4.5, 2.0, 4.5], np.float32)
    for anyhit, seed in ((False, 51), (True, 52)):
        o, d, tm, _ = scenes.random_rays(3000, lo, hi, seed=seed, anyhit_fraction=float(anyhit))
        exp = top.intersect2(o, d, tm, anyhit)
        got = restatement.trace_world(W, o, d, tm, anyhit)
        compare_queries(got, exp, sc.kind)
    px, py = restatement.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed)
    img = top.render_coords(sc, px, py)
    out = restatement.render_frame(W, sc, sc.materials, per_sample=True,
                                   specular=sc.specular, specpow=sc.specpow)
    assert out["shadow_rays"] == img["shadow_rays"]
    assert np.array_equal(out["sample_prim"], img["prim"])
    assert np.array_equal(_bits(out["sample_rgb"]), _bits(img["rgb"]))
    # spp = 1 samples the pixel centres exactly like the single-sample frame
    sc.spp = 1
    px1, py1 = restatement.sample_coords(sc.xres, sc.yres, 1, sc.seed)
    flat = restatement.primary_rays(restatement.camera_basis(sc.camera), sc.xres, sc.yres)
    img1 = top.render_coords(sc, px1, py1)
    out1 = restatement.render_frame(W, sc, sc.materials, specular=sc.specular,
                                    specpow=sc.specpow)
    assert np.array_equal(_bits(out1["rgb"]), _bits(img1["rgb"]))
    assert flat[0].shape[1] == sc.xres * sc.yres
