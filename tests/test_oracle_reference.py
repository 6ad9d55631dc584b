"""Pins the CPU restatement against the reference's own compiled classes
(oracle/_ref, built from the reference sources by oracle/ref.mk) on the full
512x512 small-frame workload: ~102k triangles, 262,144 primary rays, the
Whitted frame with hard shadows, plus random closest-hit and any-hit rays.
Skipped where the reference library was not built."""
import numpy as np
import pytest

from oracle.pyoracle import Reference

pytestmark = pytest.mark.skipif(not Reference.available(),
                                reason="oracle/_ref/libmanta_ref.so not built here")


@pytest.fixture(scope="module")
def frame():
    from rfmanta_b200 import scenes
    return scenes.small_frame_scene()


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("kind", [0, 1])
def test_small_frame_bit_exact(restatement, frame, kind):
    ref = Reference()
    rs = ref.scene(frame.mesh, kind)
    tree = rs.tree()
    assert restatement.sah_cost(tree) == pytest.approx(rs.sah_cost(), rel=0, abs=0)
    basis = ref.camera_basis(frame.camera)
    assert np.array_equal(_bits(basis), _bits(restatement.camera_basis(frame.camera)))
    org, dir = restatement.primary_rays(basis, frame.xres, frame.yres)
    tmax = np.full(org.shape[1], 1e19, np.float32)
    a = rs.intersect(org, dir, tmax)
    b = restatement.trace(tree, frame.mesh, org, dir, tmax, tri_kind=kind)
    assert np.array_equal(a["prim"], b["prim"])
    assert np.array_equal(_bits(a["t"]), _bits(b["t"]))
    img = rs.render(frame, nthreads=4)
    w = restatement.render_whitted(tree, frame, tri_kind=kind)
    assert img["shadow_rays"] == w["shadow_rays"]
    assert np.array_equal(img["prim"], w["prim"])
    assert np.array_equal(_bits(img["rgb"]), _bits(w["rgb"]))
    from rfmanta_b200 import scenes
    lo, hi = frame.mesh.bounds()
    o, d, tm, _ = scenes.random_rays(20000, lo - 0.3, hi + 0.3, seed=5, anyhit_fraction=1.0)
    x = rs.intersect(o, d, tm, anyhit=True)
    y = restatement.trace(tree, frame.mesh, o, d, tm, anyhit=True, tri_kind=kind)
    assert np.array_equal(x["hit"], y["hit"])
    rs.close()
