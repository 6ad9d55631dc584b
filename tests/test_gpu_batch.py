"""Batched multi-scene queries in one persistent, graph-captured launch:
every configuration (block size, rays per warp chunk, refill threshold,
register stack entries, node-record layout, split shared/global stack) and
the autotuned one give, for
every batch, the same bits as tracing that batch alone (rq_trace), which the
other tests tie to the reference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def setup():
    import torch
    from rfmanta_b200 import scenes
    from rfmanta_b200.batch import QueryBatch
    from rfmanta_b200.dynbvh import GpuDynBVH
    meshes = [scenes.sphere_set(3, 3, seed=1), scenes.heightfield(40, 30, seed=2, extent=4.0),
              scenes.small_frame_scene(level=3, grid=10).mesh]
    bvhs = []
    for m in meshes:
        b = GpuDynBVH()
        b.setGroup(m)
        b.rebuild()
        bvhs.append(b)
    rng = np.random.default_rng(5)
    sizes = [1, 31, 32, 33, 1000, 4097, 17, 20000, 0, 250, 3000, 64]
    batches, host = [], []
    for k, n in enumerate(sizes):
        si = int(rng.integers(0, 3))
        lo, hi = meshes[si].bounds()
        o, d, tm, _ = scenes.random_rays(n, lo - 0.3, hi + 0.3, seed=100 + k,
                                         anyhit_fraction=1.0 if k % 2 else 0.0)
        anyhit = bool(k % 2)
        if not anyhit:
            tm = np.full(n, 1e19, np.float32)
        host.append((si, o, d, tm, anyhit))
        batches.append(QueryBatch(si, torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda(),
                                  torch.from_numpy(tm).cuda(), anyhit, want_uv=True))
    return bvhs, batches, host


def _expected(bvhs, host):
    from rfmanta_b200.dynbvh import RayBatch
    out = []
    for si, o, d, tm, anyhit in host:
        r = RayBatch(o, d, tm, flags=RayBatch.AnyHit if anyhit else 0)
        if len(r):
            bvhs[si].intersect(r)
        out.append(r)
    return out


def _check(bq, exp):
    import torch
    torch.cuda.synchronize()
    for i, r in enumerate(exp):
        assert np.array_equal(bq.prim[i].cpu().numpy(), r.hitPrim), i
        assert np.array_equal(_bits(bq.t[i].cpu().numpy()), _bits(r.minT)), i


@pytest.mark.parametrize("cfg", [None,
                                 dict(block_threads=64, chunk_rays=32, refill_threshold=1, reg_stack=0),
                                 dict(block_threads=256, chunk_rays=512, refill_threshold=32, reg_stack=2),
                                 dict(block_threads=128, chunk_rays=96, refill_threshold=5, reg_stack=2,
                                      blocks_per_sm=1),
                                 dict(block_threads=128, chunk_rays=64, refill_threshold=8, reg_stack=4,
                                      node_layout=1),
                                 dict(block_threads=64, chunk_rays=128, refill_threshold=16, reg_stack=1,
                                      node_layout=2),
                                 # split stack: 2 shared entries, the rest in the overflow area
                                 dict(block_threads=256, chunk_rays=128, refill_threshold=8,
                                      smem_entries=2),
                                 dict(block_threads=96, chunk_rays=64, refill_threshold=4,
                                      smem_entries=5, node_layout=1),
                                 # split-stack kernel with a column deeper than every tree
                                 dict(block_threads=128, chunk_rays=256, refill_threshold=16,
                                      smem_entries=64, node_layout=2)])
def test_batches_match_single_queries(setup, cfg):
    from rfmanta_b200.batch import BatchedQueries
    bvhs, batches, host = setup
    bq = BatchedQueries(bvhs, batches, cfg)
    bq.launch()
    _check(bq, _expected(bvhs, host))
    bq.launch()  # graph replay
    _check(bq, _expected(bvhs, host))
    bq.close()


def test_autotune_and_new_rays(setup):
    import torch
    from rfmanta_b200.batch import BatchedQueries
    bvhs, batches, host = setup
    bq = BatchedQueries(bvhs, batches)
    cfg = bq.autotune(reps=1, candidates=[dict(chunk_rays=32), dict(chunk_rays=256, reg_stack=0)])
    assert cfg["chunk_rays"] in (32, 256)
    # the built-in search (shape, then stack entries x node layout, then
    # chunk x refill) returns a valid configuration
    full = bq.autotune(reps=1)
    assert full["reg_stack"] in (0, 1, 2, 4) and full["node_layout"] in (0, 1, 2)
    _check(bq, _expected(bvhs, host))
    # write new rays into the same device arrays and replay the plan
    rng = np.random.default_rng(9)
    for b, h in zip(batches, host):
        n = b.tmax.shape[0]
        if n:
            flip = torch.from_numpy(np.where(rng.random(n) < 0.5, -1, 1).astype(np.float32)).cuda()
            b.dir.mul_(flip)
    new_host = [(si, None, None, tm, a) for (si, o, d, tm, a) in host]
    new_host = [(si, b.org.cpu().numpy(), b.dir.cpu().numpy(), tm, a)
                for (si, _, _, tm, a), b in zip(new_host, batches)]
    bq.launch()
    _check(bq, _expected(bvhs, new_host))
    bq.close()


def test_plan_errors(setup):
    import ctypes as C
    from rfmanta_b200 import _lib
    bvhs, batches, host = setup
    arr = (_lib.Batch * 1)()
    arr[0].scene = 5
    arr[0].n = 1
    arr[0].flags = 0
    scenes = (C.c_void_p * 1)(bvhs[0].handle.value)
    plan = C.c_void_p()
    assert _lib.lib.rq_batch_plan_create(scenes, 1, arr, 1, None, C.byref(plan)) == _lib.RQ_ERR_ARG
    arr[0].scene = 0
    assert _lib.lib.rq_batch_plan_create(scenes, 1, arr, 1, None, C.byref(plan)) == _lib.RQ_ERR_ARG
    b = batches[0]
    arr[0].n = int(b.tmax.shape[0])
    arr[0].d_org, arr[0].d_dir, arr[0].d_tmax = b.org.data_ptr(), b.dir.data_ptr(), b.tmax.data_ptr()
    for bad in (dict(smem_entries=65), dict(smem_entries=-1), dict(smem_entries=8, reg_stack=2)):
        cfg = _lib.BatchConfig(block_threads=128, chunk_rays=128, refill_threshold=8, **bad)
        assert _lib.lib.rq_batch_plan_create(scenes, 1, arr, 1, C.byref(cfg),
                                             C.byref(plan)) == _lib.RQ_ERR_ARG, bad


def test_plan_follows_scene_updates():
    """A plan made before a scene's mesh moved (rotating update, new tree
    layout, possibly a deeper tree) launches on the updated scene: the plan
    copies in the scene's new descriptor, and its results equal tracing the
    updated scene alone."""
    import torch
    from rfmanta_b200 import scenes
    from rfmanta_b200.batch import BatchedQueries, QueryBatch
    from rfmanta_b200.dynbvh import GpuDynBVH
    mesh = scenes.small_frame_scene(level=3, grid=10).mesh
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.rebuild()
    lo, hi = mesh.bounds()
    o, d, tm, _ = scenes.random_rays(5000, lo - 0.3, hi + 0.3, seed=3)
    tm = np.full(o.shape[1], 1e19, np.float32)
    batch = QueryBatch(0, torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda(),
                       torch.from_numpy(tm).cuda(), False, want_uv=True)
    bq = BatchedQueries([bvh], [batch], dict(reg_stack=0))
    bq.launch()
    # a plan over a breadth-first copy of the records follows the updates too
    bq2 = BatchedQueries([bvh], [batch], dict(reg_stack=2, node_layout=1))
    # and a split-stack plan, whose overflow area grows with a deeper tree
    bq3 = BatchedQueries([bvh], [batch], dict(smem_entries=3))
    v0 = mesh.vertices.copy()
    for k, rotate in ((1, True), (2, False), (3, True)):
        mesh.vertices = scenes.animated_vertices(v0, k, amplitude=0.05)
        bvh.update(rotate=rotate)
        for p in (bq, bq2, bq3):
            p.launch()
            _check(p, _expected([bvh], [(0, o, d, tm, False)]))
    bq.close()
    bq2.close()
    bq3.close()


@pytest.mark.parametrize("cfg", [dict(block_threads=128, chunk_rays=64, refill_threshold=8),
                                 dict(block_threads=256, chunk_rays=128, refill_threshold=16,
                                      smem_entries=3, node_layout=1)])
def test_kensler_shirley_batches_match_single_queries(cfg):
    """The same check with Kensler-Shirley triangle records (the plan's
    kernels are compiled per triangle kind), whole stack in shared memory
    and split."""
    import torch
    from rfmanta_b200 import scenes
    from rfmanta_b200.batch import BatchedQueries, QueryBatch
    from rfmanta_b200.dynbvh import GpuDynBVH
    meshes = [scenes.sphere_set(2, 3, seed=4), scenes.heightfield(30, 30, seed=5, extent=3.0)]
    bvhs = []
    for m in meshes:
        b = GpuDynBVH(tri_kind=1)
        b.setGroup(m)
        b.rebuild()
        bvhs.append(b)
    batches, host = [], []
    for k, n in enumerate([700, 33, 5000, 1]):
        si = k % 2
        lo, hi = meshes[si].bounds()
        anyhit = bool(k % 2)
        o, d, tm, _ = scenes.random_rays(n, lo - 0.3, hi + 0.3, seed=300 + k,
                                         anyhit_fraction=1.0 if anyhit else 0.0)
        if not anyhit:
            tm = np.full(n, 1e19, np.float32)
        host.append((si, o, d, tm, anyhit))
        batches.append(QueryBatch(si, torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda(),
                                  torch.from_numpy(tm).cuda(), anyhit, want_uv=True))
    bq = BatchedQueries(bvhs, batches, cfg)
    bq.launch()
    _check(bq, _expected(bvhs, host))
    bq.close()
    for b in bvhs:
        b.close()
