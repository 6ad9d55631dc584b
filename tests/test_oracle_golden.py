"""The CPU restatement (oracle/rq_oracle.c) against the golden vectors the
reference itself produced (tests/golden/make_golden.py)."""
import numpy as np

from conftest import golden_mesh, golden_tree

KIND = {"wald": 0, "ks": 1}


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _same(a, b):
    return np.array_equal(_bits(a), _bits(b))


def test_sah_cost_matches_reference(restatement, golden):
    _, g = golden
    assert restatement.sah_cost(golden_tree(g)) == float(np.float32(g["sah_cost"]))


def test_camera_basis_matches_reference(restatement, golden):
    from rfmanta_b200.scenes import Camera
    _, g = golden
    c = g["cam"]
    cam = Camera(tuple(c[0:3]), tuple(c[3:6]), tuple(c[6:9]), float(c[9]), float(c[10]))
    assert _same(restatement.camera_basis(cam), g["camera_basis"])


def test_primary_rays_match(restatement, golden):
    _, g = golden
    org, dir = restatement.primary_rays(g["camera_basis"], int(g["xres"]), int(g["yres"]))
    assert _same(org, g["primary_org"]) and _same(dir, g["primary_dir"])


def _check_query(restatement, g, kind, prefix, tmax, anyhit):
    org, dir = g[f"{prefix}_org"], g[f"{prefix}_dir"]
    out = restatement.trace(golden_tree(g), golden_mesh(g), org, dir, tmax, anyhit=anyhit,
                            tri_kind=KIND[kind])
    assert np.array_equal(out["hit"], g[f"{prefix}_hit"])
    if anyhit:
        return
    hit = g[f"{prefix}_hit"] > 0
    assert np.array_equal(out["prim"], g[f"{prefix}_prim"])
    assert _same(out["t"], g[f"{prefix}_t"])
    assert _same(out["u"][hit], g[f"{prefix}_u"][hit])
    assert _same(out["v"][hit], g[f"{prefix}_v"][hit])


def test_primary_closest_hits(restatement, golden):
    kind, g = golden
    n = g["primary_org"].shape[1]
    _check_query(restatement, g, kind, "primary", np.full(n, 1e19, np.float32), False)


def test_random_closest_hits(restatement, golden):
    kind, g = golden
    n = g["rand_org"].shape[1]
    _check_query(restatement, g, kind, "rand", np.full(n, 1e19, np.float32), False)


def test_random_anyhit(restatement, golden):
    kind, g = golden
    _check_query(restatement, g, kind, "any", g["any_tmax"], True)


def test_whitted_frame(restatement, golden):
    from rfmanta_b200.scenes import Camera, PointLightSpec, WhittedScene
    kind, g = golden
    c = g["cam"]
    cam = Camera(tuple(c[0:3]), tuple(c[3:6]), tuple(c[6:9]), float(c[9]), float(c[10]))
    lights = [PointLightSpec(tuple(l[:3]), tuple(l[3:])) for l in g["lights"]]
    sc = WhittedScene(golden_mesh(g), cam, lights, tuple(g["ambient"]), tuple(g["background"]),
                      int(g["xres"]), int(g["yres"]))
    out = restatement.render_whitted(golden_tree(g), sc, tri_kind=KIND[kind])
    assert out["shadow_rays"] == int(g["img_shadow_rays"])
    assert np.array_equal(out["prim"], g["img_prim"])
    assert _same(out["t"], g["img_t"])
    assert _same(out["rgb"], g["img_rgb"])


def test_blob_layout_is_reference_layout(golden):
    """The saveToFile stream parses into the same fields the reference holds."""
    from rfmanta_b200.treeio import parse_dynbvh_blob
    _, g = golden
    assert int(g["node_size"]) == 32
    t = parse_dynbvh_blob(g["blob"].tobytes(), n_tris=g["indices"].shape[0])
    n = g["bounds"].shape[0]
    assert np.array_equal(t.bounds[:n], g["bounds"])
    assert np.array_equal(t.child[:n], g["child"])
    assert np.array_equal(t.children[:n], g["children"])
    assert np.array_equal(t.axis[:n], g["axis"])
    assert np.array_equal(t.left_cheaper[:n], g["left_cheaper"])
    assert np.array_equal(t.ids, g["ids"])


def test_sincos_2pi_error_bound(restatement):
    """The path tracer's own sin/cos of 2*pi*u (quadrant reduction + Taylor
    polynomials) stays within 2e-7 of the exact values over [0, 1)."""
    u = np.concatenate([np.linspace(0, 1, 200001, endpoint=False, dtype=np.float32),
                        np.random.default_rng(0).random(100000).astype(np.float32)])
    c, s = restatement.sincos_2pi(u)
    a = 2 * np.pi * u.astype(np.float64)
    assert np.max(np.abs(c - np.cos(a))) < 2e-7
    assert np.max(np.abs(s - np.sin(a))) < 2e-7
