"""The C++ drop-in: the reference's own Raytracer + Lambertian + HardShadows
(compiled from the reference sources) rendering through GpuDynBVH, the
AccelerationStructure backed by the CUDA library, against the same frame
rendered through the reference's DynBVH.  With the reference tree imported
through DynBVH::saveToFile / GpuDynBVH::buildFromFile the frames are equal
bit for bit; with the drop-in's own GPU-built tree only pixels whose nearest
hits tie may differ."""
import os

import numpy as np
import pytest

from oracle.pyoracle import DROPIN_SO, Reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(DROPIN_SO),
                                 reason="oracle/_ref/libmanta_dropin.so not built")]


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("kind", [0, 1])
def test_raytracer_through_gpu_dynbvh(kind, tmp_path):
    from rfmanta_b200 import scenes
    sc = scenes.small_frame_scene(xres=256, yres=256)
    ref = Reference(path=DROPIN_SO)
    cpu = ref.scene(sc.mesh, kind)
    want = cpu.render(sc, nthreads=4)
    gpu = ref.scene(sc.mesh, kind)
    gpu.use_gpu(0, kind, tree_file=str(tmp_path / "tree.bvh"))
    got = gpu.render(sc, nthreads=4)
    assert got["shadow_rays"] == want["shadow_rays"]
    assert np.array_equal(got["prim"], want["prim"])
    assert np.array_equal(_bits(got["rgb"]), _bits(want["rgb"]))
    # any-hit and closest-hit packets through the drop-in
    lo, hi = sc.mesh.bounds()
    o, d, tm, _ = scenes.random_rays(5000, lo - 0.2, hi + 0.2, seed=3, anyhit_fraction=1.0)
    a = cpu.intersect(o, d, tm, anyhit=True)
    b = gpu.intersect(o, d, tm, anyhit=True)
    assert np.array_equal(a["hit"], b["hit"])
    own = ref.scene(sc.mesh, kind)
    own.use_gpu(0, kind)  # GPU-built tree
    img = own.render(sc, nthreads=4)
    differ = (img["prim"] != want["prim"]).mean()
    assert differ < 1e-3, differ


@pytest.mark.parametrize("kind", [0, 1])
def test_gpu_hard_shadows_and_batched_packets(kind, tmp_path):
    """GpuHardShadows (all lights' shadow rays of a packet in one
    submission), the submission queue (concurrent workers' packets gathered
    into batches) and the resident packet channel under the reference's own
    Raytracer and Lambertian, with three point lights and 32 worker threads:
    the frame, the per-pixel hits and the shadow-ray count equal the
    reference's DynBVH + HardShadows render bit for bit in every packet
    mode."""
    from rfmanta_b200 import scenes
    sc = scenes.small_frame_scene(xres=192, yres=160)
    sc.lights = list(sc.lights) + [scenes.PointLightSpec((-2.5, 2.0, 1.0), (0.3, 0.35, 0.4)),
                                   scenes.PointLightSpec((0.0, -3.0, 0.5), (0.2, 0.2, 0.2))]
    ref = Reference(path=DROPIN_SO)
    cpu = ref.scene(sc.mesh, kind)
    want = cpu.render(sc, nthreads=8)
    gpu = ref.scene(sc.mesh, kind)
    gpu.use_gpu(0, kind, tree_file=str(tmp_path / "tree.bvh"))
    # packet modes: 0 one round trip per call, 1 submission queue, 2 resident channel
    for mode, gpu_shadows in ((1, True), (0, True), (1, False), (2, True), (2, False)):
        gpu.gpu_options(mode=mode, gpu_shadows=gpu_shadows)
        got = gpu.render(sc, nthreads=32)
        assert got["shadow_rays"] == want["shadow_rays"], (mode, gpu_shadows)
        assert np.array_equal(got["prim"], want["prim"]), (mode, gpu_shadows)
        assert np.array_equal(_bits(got["rgb"]), _bits(want["rgb"])), (mode, gpu_shadows)


def test_gpu_mesh_as_primitive_in_a_group(tmp_path):
    """The Primitive surface: a reference Group holding one GpuMeshPrimitive
    over the drop-in, traced through Group::intersect, renders the frame of
    the reference's DynBVH bit for bit (with HardShadows and with
    GpuHardShadows)."""
    from rfmanta_b200 import scenes
    sc = scenes.small_frame_scene(xres=160, yres=128)
    ref = Reference(path=DROPIN_SO)
    cpu = ref.scene(sc.mesh, 0)
    want = cpu.render(sc, nthreads=4)
    gpu = ref.scene(sc.mesh, 0)
    gpu.use_gpu(0, 0, tree_file=str(tmp_path / "tree.bvh"))
    gpu.gpu_as_primitive()
    for gpu_shadows in (False, True):
        gpu.gpu_options(batching=True, gpu_shadows=gpu_shadows)
        got = gpu.render(sc, nthreads=8)
        assert got["shadow_rays"] == want["shadow_rays"]
        assert np.array_equal(got["prim"], want["prim"])
        assert np.array_equal(_bits(got["rgb"]), _bits(want["rgb"]))
