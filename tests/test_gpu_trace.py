"""Device traversal (closest hit / any hit, Wald and Kensler-Shirley) through
the C ABI, against the reference's golden vectors and the CPU restatement.

Integer results (hit flag, triangle id) and float results (t, u, v) are
compared bit for bit: the device path uses the reference's float operation
order with no fused multiply-add, so no tolerance is needed."""
import threading

import numpy as np
import pytest

from conftest import golden_mesh, golden_tree, has_gpu

pytestmark = pytest.mark.gpu

KIND = {"wald": 0, "ks": 1}


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _bvh(mesh, kind, tree=None, blob=None):
    from rfmanta_b200.dynbvh import GpuDynBVH
    b = GpuDynBVH(tri_kind=kind)
    b.setGroup(mesh)
    if blob is not None:
        b.importBlob(blob)
    else:
        b.importTree(tree)
    return b


def _query(bvh, org, dir, tmax, anyhit=False):
    from rfmanta_b200.dynbvh import RayBatch
    rays = RayBatch(org, dir, tmax, flags=RayBatch.AnyHit if anyhit else 0)
    bvh.intersect(rays)
    return rays


def _assert_matches_golden(g, prefix, rays, anyhit):
    hit = g[f"{prefix}_hit"] > 0
    assert np.array_equal(rays.wasHit(), hit)
    if anyhit:
        return
    assert np.array_equal(rays.hitPrim, g[f"{prefix}_prim"])
    assert np.array_equal(_bits(rays.minT), _bits(g[f"{prefix}_t"]))
    assert np.array_equal(_bits(rays.u[hit]), _bits(g[f"{prefix}_u"][hit]))
    assert np.array_equal(_bits(rays.v[hit]), _bits(g[f"{prefix}_v"][hit]))


@pytest.mark.parametrize("source", ["fields", "blob"])
def test_golden_queries(golden, source):
    kind, g = golden
    mesh = golden_mesh(g)
    bvh = _bvh(mesh, KIND[kind], tree=golden_tree(g),
               blob=g["blob"].tobytes() if source == "blob" else None)
    n = g["primary_org"].shape[1]
    r = _query(bvh, g["primary_org"], g["primary_dir"], np.full(n, 1e19, np.float32))
    _assert_matches_golden(g, "primary", r, False)
    n = g["rand_org"].shape[1]
    r = _query(bvh, g["rand_org"], g["rand_dir"], np.full(n, 1e19, np.float32))
    _assert_matches_golden(g, "rand", r, False)
    r = _query(bvh, g["any_org"], g["any_dir"], g["any_tmax"], anyhit=True)
    _assert_matches_golden(g, "any", r, True)
    assert bvh.sahCost() == float(np.float32(g["sah_cost"]))


@pytest.mark.parametrize("persistent,block,refill", [(False, 128, 1), (True, 128, 1),
                                                     (True, 64, 8), (True, 256, 32)])
def test_launch_forms_agree(golden, persistent, block, refill):
    kind, g = golden
    bvh = _bvh(golden_mesh(g), KIND[kind], tree=golden_tree(g))
    for anyhit in (False, True):
        bvh.set_launch_config(anyhit, block_threads=block, refill_threshold=refill,
                              persistent=persistent)
    n = g["rand_org"].shape[1]
    r = _query(bvh, g["rand_org"], g["rand_dir"], np.full(n, 1e19, np.float32))
    _assert_matches_golden(g, "rand", r, False)
    r = _query(bvh, g["any_org"], g["any_dir"], g["any_tmax"], anyhit=True)
    _assert_matches_golden(g, "any", r, True)


def test_export_roundtrip(golden):
    from rfmanta_b200.treeio import parse_dynbvh_blob
    kind, g = golden
    bvh = _bvh(golden_mesh(g), KIND[kind], blob=g["blob"].tobytes())
    t = parse_dynbvh_blob(bvh.exportBlob())
    n = g["bounds"].shape[0]
    assert np.array_equal(t.bounds[:n], g["bounds"])
    assert np.array_equal(t.child[:n], g["child"])
    assert np.array_equal(t.children[:n], g["children"])
    assert np.array_equal(t.ids, g["ids"])


def test_empty_and_single_ray(golden):
    kind, g = golden
    bvh = _bvh(golden_mesh(g), KIND[kind], tree=golden_tree(g))
    r = _query(bvh, np.zeros((3, 0), np.float32), np.zeros((3, 0), np.float32),
               np.zeros(0, np.float32))
    assert len(r) == 0
    o = g["rand_org"][:, :1].copy()
    d = g["rand_dir"][:, :1].copy()
    r = _query(bvh, o, d, np.full(1, 1e19, np.float32))
    assert r.hitPrim[0] == g["rand_prim"][0]


def test_edge_rays_match_restatement(restatement):
    """Axis-parallel directions (infinite inverse), zero-length tmax, origins
    on box faces and inside the mesh, a degenerate triangle."""
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    m = scenes.small_frame_scene(level=2, grid=4).mesh
    # add a zero-area triangle
    v = np.concatenate([m.vertices, np.array([[0.1, 0.2, 0.3]] * 3, np.float32)])
    nv = m.vertices.shape[0]
    ix = np.concatenate([m.indices, np.array([[nv, nv + 1, nv + 2]], np.uint32)])
    fm = np.concatenate([m.face_material, np.zeros(1, np.uint32)])
    mesh = scenes.Mesh(v, ix, fm, m.materials)
    from oracle.pyoracle import Reference
    rng = np.random.default_rng(3)
    n = 3000
    o = rng.uniform(-1.5, 1.5, (3, n)).astype(np.float32)
    d = rng.normal(size=(3, n)).astype(np.float32)
    d[:, :600] = 0.0
    d[rng.integers(0, 3, 600), np.arange(600)] = rng.choice([-1.0, 1.0], 600)
    d[0, 600:900] = 0.0
    o[:, 900:1000] = 0.0  # inside the sphere
    o[1, 1000:1100] = -1.1  # on the ground plane
    tmax = np.full(n, 1e19, np.float32)
    tmax[1100:1200] = 0.0
    tmax[1200:1300] = 1e-5
    for kind in (0, 1):
        if Reference.available():
            tree = Reference().scene(mesh, kind).tree()
        else:
            pytest.skip("needs a reference-built tree")
        bvh = GpuDynBVH(tri_kind=kind)
        bvh.setGroup(mesh)
        bvh.importTree(tree)
        for anyhit in (False, True):
            exp = restatement.trace(tree, mesh, o, d, tmax, anyhit=anyhit, tri_kind=kind)
            r = _query(bvh, o, d, tmax, anyhit=anyhit)
            assert np.array_equal(r.wasHit(), exp["hit"] > 0)
            if not anyhit:
                assert np.array_equal(r.hitPrim, exp["prim"])
                assert np.array_equal(_bits(r.minT), _bits(exp["t"]))


def test_full_small_frame_matches_restatement(restatement):
    """512x512 primary rays over the ~102k-triangle scene, both triangle
    kinds, every ray bit-exact against the restatement on the same tree."""
    from oracle.pyoracle import Reference
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    if not Reference.available():
        pytest.skip("needs a reference-built tree")
    sc = scenes.small_frame_scene()
    basis = restatement.camera_basis(sc.camera)
    org, dir = restatement.primary_rays(basis, sc.xres, sc.yres)
    tmax = np.full(org.shape[1], 1e19, np.float32)
    for kind in (0, 1):
        tree = Reference().scene(sc.mesh, kind).tree()
        bvh = GpuDynBVH(tri_kind=kind)
        bvh.setGroup(sc.mesh)
        bvh.importTree(tree)
        exp = restatement.trace(tree, sc.mesh, org, dir, tmax, tri_kind=kind)
        r = _query(bvh, org, dir, tmax)
        assert np.array_equal(r.hitPrim, exp["prim"])
        assert np.array_equal(_bits(r.minT), _bits(exp["t"]))
        hit = exp["hit"] > 0
        assert np.array_equal(_bits(r.u[hit]), _bits(exp["u"][hit]))


def test_errors_are_reported(golden):
    from rfmanta_b200 import _lib
    from rfmanta_b200.dynbvh import GpuDynBVH, RayBatch
    kind, g = golden
    bvh = GpuDynBVH(tri_kind=KIND[kind])
    bvh.setGroup(golden_mesh(g))
    bvh._upload()
    with pytest.raises(_lib.RQError) as e:
        bvh.intersect(RayBatch(g["rand_org"], g["rand_dir"]))
    assert e.value.code == _lib.RQ_ERR_STATE
    blob = bytearray(g["blob"].tobytes())
    with pytest.raises(_lib.RQError) as e:
        bvh.importBlob(bytes(blob[:100]))
    assert e.value.code == _lib.RQ_ERR_FORMAT
    # point the root's child at itself: a cycle
    nids = int(np.frombuffer(bytes(blob[:4]), "<u4")[0])
    off = 4 + 4 * nids + 4
    blob[off + 24:off + 28] = np.int32(0).tobytes()
    blob[off + 30:off + 32] = np.int16(0).tobytes()
    with pytest.raises(_lib.RQError) as e:
        bvh.importBlob(bytes(blob))
    assert e.value.code == _lib.RQ_ERR_FORMAT
    # the scene stays usable after the errors
    bvh.importBlob(g["blob"].tobytes())
    n = g["rand_org"].shape[1]
    r = _query(bvh, g["rand_org"], g["rand_dir"], np.full(n, 1e19, np.float32))
    _assert_matches_golden(g, "rand", r, False)


def test_concurrent_callers(golden):
    """Several host threads calling intersect on one scene at once (the
    reference calls DynBVH::intersect from every render worker)."""
    kind, g = golden
    bvh = _bvh(golden_mesh(g), KIND[kind], tree=golden_tree(g))
    n = g["rand_org"].shape[1]
    errs = []

    def work(k):
        try:
            for _ in range(5):
                sl = slice(k * 256, (k + 1) * 256)
                r = _query(bvh, g["rand_org"][:, sl].copy(), g["rand_dir"][:, sl].copy(),
                           np.full(256, 1e19, np.float32))
                assert np.array_equal(r.hitPrim, g["rand_prim"][sl])
        except Exception as ex:  # pragma: no cover
            errs.append(ex)

    th = [threading.Thread(target=work, args=(k,)) for k in range(8)]
    [t.start() for t in th]
    [t.join() for t in th]
    assert not errs, errs
