"""rq_render_whitted_device_noalloc, the Whitted frame for callers that
cannot allocate device memory (a process whose device memory belongs to
another allocator, a render thread that must not make device-synchronising
calls such as cudaMalloc).  Its scratch is a fixed array inside the library,
so it is checked here against the allocating entry point
rq_render_whitted_device: two calls in a row, each equal to the allocating
call bit for bit (the tolerance all frame tests use: none), and no change in
free device memory from before the first no-alloc call to after the second.
A threaded test runs no-alloc frames beside tree updates of the same scene
on another host thread.  The file name makes pytest collect it last."""
import ctypes as C
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_noalloc_frame_matches_allocating_entry_point():
    import torch
    from rfmanta_b200 import _lib, scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.small_frame_scene()
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    p = bvh.whitted_params(sc)
    npx = sc.xres * sc.yres
    stream = torch.cuda.current_stream().cuda_stream

    def buffers():
        return (torch.zeros(npx * 3, device="cuda"), torch.zeros(npx, device="cuda"),
                torch.zeros(npx, dtype=torch.int32, device="cuda"),
                torch.zeros(1, dtype=torch.int64, device="cuda"))

    want = buffers()
    _lib.check(_lib.lib.rq_render_whitted_device(
        bvh.handle, C.byref(p), C.c_void_p(want[0].data_ptr()), C.c_void_p(want[1].data_ptr()),
        C.c_void_p(want[2].data_ptr()), C.c_void_p(want[3].data_ptr()), C.c_void_p(stream)))
    torch.cuda.synchronize()
    outs = [buffers(), buffers()]
    torch.cuda.synchronize()
    free = [torch.cuda.mem_get_info()[0]]
    for got in outs:
        _lib.check(_lib.lib.rq_render_whitted_device_noalloc(
            bvh.handle, C.byref(p), C.c_void_p(got[0].data_ptr()),
            C.c_void_p(got[1].data_ptr()), C.c_void_p(got[2].data_ptr()),
            C.c_void_p(got[3].data_ptr()), C.c_void_p(stream)))
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    for got in outs:
        assert int(got[3].item()) == int(want[3].item())
        assert np.array_equal(got[2].cpu().numpy(), want[2].cpu().numpy())
        assert np.array_equal(_bits(got[1].cpu().numpy()), _bits(want[1].cpu().numpy()))
        assert np.array_equal(_bits(got[0].cpu().numpy()), _bits(want[0].cpu().numpy()))
    assert free[1] == free[0] and free[2] == free[0], free


def test_noalloc_large_frames_and_material_limit():
    """The frame kernel keeps no per-pixel scratch, so a 2048x1024 frame
    renders through the fixed array as through the allocating entry point;
    a material table beyond the array's 1,024 entries is refused."""
    import torch
    from rfmanta_b200 import _lib, scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.small_frame_scene(level=2, grid=4, xres=2048, yres=1024)
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    p = bvh.whitted_params(sc)
    npx = sc.xres * sc.yres
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    outs = []
    for fn in (_lib.lib.rq_render_whitted_device, _lib.lib.rq_render_whitted_device_noalloc):
        rgb = torch.zeros(npx * 3, device="cuda")
        t = torch.zeros(npx, device="cuda")
        prim = torch.zeros(npx, dtype=torch.int32, device="cuda")
        _lib.check(fn(bvh.handle, C.byref(p), C.c_void_p(rgb.data_ptr()),
                      C.c_void_p(t.data_ptr()), C.c_void_p(prim.data_ptr()), None, stream))
        torch.cuda.synchronize()
        outs.append((rgb.cpu().numpy(), prim.cpu().numpy()))
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(_bits(outs[0][0]), _bits(outs[1][0]))
    mats = np.full((1025, 3), 0.5, np.float32)
    p.n_materials = mats.shape[0]
    p.material_rgb = mats.ctypes.data
    tiny = torch.zeros(npx * 3, device="cuda")
    rc = _lib.lib.rq_render_whitted_device_noalloc(bvh.handle, C.byref(p),
                                                   C.c_void_p(tiny.data_ptr()),
                                                   C.c_void_p(tiny.data_ptr()),
                                                   C.c_void_p(tiny.data_ptr()), None, None)
    assert rc == _lib.RQ_ERR_CAPACITY
    assert b"materials" in _lib.lib.rq_last_error()


def test_noalloc_frames_beside_updates_on_another_thread():
    """Manta's workers call into one scene from several host threads.  One
    thread renders no-alloc frames while another updates the same scene's
    tree (with rotations, which can replace the node records); both use the
    legacy default stream, so the GPU runs their work in launch order, and
    the scene's lock keeps every frame's snapshot of the tree valid.  After
    both finish, the no-alloc frame equals the allocating one."""
    import torch
    from rfmanta_b200 import _lib, scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = scenes.small_frame_scene(level=4, grid=30, xres=256, yres=256)
    bvh = GpuDynBVH()
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    p = bvh.whitted_params(sc)
    npx = sc.xres * sc.yres
    v0 = sc.mesh.vertices.copy()
    poses = [np.ascontiguousarray(scenes.wave_vertices(v0, k, 4)) for k in range(4)]
    rgb = torch.zeros(npx * 3, device="cuda")
    t = torch.zeros(npx, device="cuda")
    prim = torch.zeros(npx, dtype=torch.int32, device="cuda")
    errors = []

    def frames():
        for _ in range(40):
            rc = _lib.lib.rq_render_whitted_device_noalloc(
                bvh.handle, C.byref(p), C.c_void_p(rgb.data_ptr()), C.c_void_p(t.data_ptr()),
                C.c_void_p(prim.data_ptr()), None, None)
            if rc != _lib.RQ_OK:
                errors.append(("frame", rc))

    def updates():
        for k in range(40):
            v = poses[k % 4]
            rc = _lib.lib.rq_scene_update_vertices_ex(bvh.handle, C.c_void_p(v.ctypes.data),
                                                      v.shape[0], _lib.RQ_UPDATE_ROTATE)
            if rc != _lib.RQ_OK:
                errors.append(("update", rc))

    th = [threading.Thread(target=frames), threading.Thread(target=updates)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    torch.cuda.synchronize()
    assert not errors, errors
    outs = []
    for fn in (_lib.lib.rq_render_whitted_device, _lib.lib.rq_render_whitted_device_noalloc):
        o = (torch.zeros(npx * 3, device="cuda"), torch.zeros(npx, dtype=torch.int32, device="cuda"))
        _lib.check(fn(bvh.handle, C.byref(p), C.c_void_p(o[0].data_ptr()),
                      C.c_void_p(t.data_ptr()), C.c_void_p(o[1].data_ptr()), None, None))
        torch.cuda.synchronize()
        outs.append((o[0].cpu().numpy(), o[1].cpu().numpy()))
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(_bits(outs[0][0]), _bits(outs[1][0]))
    assert (outs[1][1] >= 0).any()
