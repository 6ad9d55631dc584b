"""EyeAmbient and LinearBackground on the CPU: the restatement (oracle/
rq_oracle.c env_ambient / env_background) against the reference's
EyeAmbient::computeAmbient (Model/AmbientLights/EyeAmbient.cc:29-44) and
LinearBackground::shade (Model/Backgrounds/LinearBackground.cc:28-40) as its
Raytracer, Phong reflection recursion and KajiyaPathtracer use them.

Pinned by tests/golden/tiny_env.npz: a Whitted frame and a reflective Phong
frame bit for bit per pixel / sample, and path-traced images in expectation
(the path tracer's EyeAmbient at the last bounce sees the direction
sampleBSDF wrote into the packet and face-forward normals recomputed
against it, which the statistics check)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def load_env():
    z = np.load(os.path.join(GOLDEN, "tiny_env.npz"))
    return {k: z[k] for k in z.files}


def _golden_dir():
    import sys
    if GOLDEN not in sys.path:
        sys.path.insert(0, GOLDEN)


def env_tree(g):
    from oracle.pyoracle import Tree
    return Tree(*[g[f"tree_{f}"] for f in ("bounds", "child", "children", "axis",
                                           "left_cheaper", "ids")])


def whitted_case():
    """(scene, environment) of the fixture's Whitted frame."""
    _golden_dir()
    from make_golden import environment
    from rfmanta_b200 import scenes
    sc = scenes.tiny_frame_scene(xres=48, yres=40)
    sc.environment = environment()
    return sc


def test_whitted_fixture(restatement):
    g = load_env()
    sc = whitted_case()
    out = restatement.render_whitted(env_tree(g), sc)
    assert out["shadow_rays"] == int(g["whitted_shadow_rays"])
    assert np.array_equal(out["prim"], g["whitted_prim"])
    assert np.array_equal(_bits(out["t"]), _bits(g["whitted_t"]))
    assert np.array_equal(_bits(out["rgb"]), _bits(g["whitted_rgb"]))
    miss = out["prim"] < 0
    assert miss.sum() > 100  # the background gradient is on screen
    assert len(np.unique(out["rgb"][miss], axis=0)) > 50
    sc.environment = None
    plain = restatement.render_whitted(env_tree(g), sc)
    assert np.all((plain["rgb"] != out["rgb"]).any(1))  # every pixel changed


def test_reflective_frame_fixture(restatement):
    _golden_dir()
    from make_golden import REFLECT
    g = load_env()
    sc = whitted_case()
    sc.xres, sc.yres, sc.spp, sc.seed = 40, 32, 4, 5
    m = sc.mesh
    n = m.materials.shape[0]
    W = restatement.world(env_tree(g), m)
    out = restatement.render_frame(W, sc, m.materials, per_sample=True,
                                   specular=np.full((n, 3), 0.4, np.float32),
                                   specpow=np.array(REFLECT["flat_specpow"][:n], np.int32),
                                   reflectivity=np.array(REFLECT["flat_refl"][:n], np.float32))
    assert out["shadow_rays"] == int(g["frame_shadow_rays"])
    assert np.array_equal(out["sample_prim"], g["frame_sample_prim"])
    assert np.array_equal(_bits(out["sample_rgb"]), _bits(g["frame_sample_rgb"]))


def path_case(depth):
    _golden_dir()
    from make_golden import ENVIRONMENT, PATH_STATS, environment
    from rfmanta_b200 import scenes
    p = PATH_STATS
    sc = scenes.tiny_path_scene(xres=p["xres"], yres=p["yres"], spp=p["spp"])
    sc.ambient, sc.background = ENVIRONMENT["path_ambient"], ENVIRONMENT["path_background"]
    sc.max_depth = depth
    sc.environment = environment()
    return sc


@pytest.mark.parametrize("depth", [1, 2])
def test_path_images_match_reference_in_expectation(restatement, depth):
    """At depth 1 every hit path is at its last bounce, so the EyeAmbient
    term dominates: reading the incoming direction and its normal there
    instead of the sampled direction puts the image means 49-95 standard
    errors off.  At depth 2 bounce rays also reach the LinearBackground."""
    from test_oracle_path_stats import _median_tree, _ours, _z
    g = load_env()
    ref = g[f"path_images_d{depth}"].astype(np.float64)
    sc = path_case(depth)
    tree = _median_tree(sc.mesh)
    ours = _ours(restatement, tree, sc, range(7000, 7000 + ref.shape[0]))
    img_z = _z(ours.mean((1, 2)), ref.mean((1, 2)))
    assert np.all(np.abs(img_z) < 4.0), img_z
    pix_z = _z(ours, ref)
    assert abs(pix_z.mean()) < 0.3, pix_z.mean()
    assert np.mean(np.abs(pix_z) > 4.0) < 0.01
    # the check sees a 0.1% bias, and the constant forms are far off
    biased = _z((ours * 1.001).mean((1, 2)), ref.mean((1, 2)))
    assert np.all(np.abs(biased) > 4.0), biased
    sc.environment = None  # (cup and cdown share their green)
    flat = _ours(restatement, tree, sc, range(8000, 8008))
    assert np.abs(_z(flat.mean((1, 2)), ref.mean((1, 2)))).max() > 8.0


@pytest.mark.parametrize("ambient,background", [("eye", "constant"), ("constant", "linear")])
def test_live_reference_whitted(restatement, ambient, background):
    """Each form on its own, live, with an unnormalised up vector."""
    from oracle.pyoracle import Reference
    from rfmanta_b200 import scenes
    if not Reference.available():
        pytest.skip("reference library not built")
    ref = Reference()
    env = scenes.Environment(ambient=ambient, background=background,
                             background_down=(0.05, 0.6, 0.2), background_up=(-3.0, 2.0, 0.5))
    sc = scenes.tiny_frame_scene(xres=32, yres=24)
    sc.environment = env
    rs = ref.scene(sc.mesh, 0)
    rs.set_environment(env)
    img = rs.render(sc)
    out = restatement.render_whitted(rs.tree(), sc)
    rs.close()
    assert out["shadow_rays"] == img["shadow_rays"]
    assert np.array_equal(_bits(out["rgb"]), _bits(img["rgb"]))
