"""Batched ray queries over several resident scenes (the batched form).

``BatchedQueries`` owns the per-batch output buffers (torch tensors on the
scenes' device), builds an ``rq_batch`` table, creates a graph-captured plan
and launches it; ``autotune`` picks the launch configuration with the
library's own autotuner (rq_batch_autotune)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib
from ._lib import check, lib


@dataclass
class QueryBatch:
    scene: int          # index into the scene list
    org: object         # torch (3, n) float32 cuda, contiguous
    dir: object         # torch (3, n) float32 cuda
    tmax: object        # torch (n,) float32 cuda
    anyhit: bool = False
    want_uv: bool = False


class BatchedQueries:
    def __init__(self, scenes, batches: list[QueryBatch], config: dict | None = None):
        import torch
        self.scenes = scenes
        self.batches = batches
        dev = batches[0].org.device
        self.t = [torch.empty(b.tmax.shape[0], device=dev) for b in batches]
        self.prim = [torch.empty(b.tmax.shape[0], dtype=torch.int32, device=dev) for b in batches]
        self.u = [torch.empty(b.tmax.shape[0], device=dev) if b.want_uv else None for b in batches]
        self.v = [torch.empty(b.tmax.shape[0], device=dev) if b.want_uv else None for b in batches]
        self._scene_arr = (C.c_void_p * len(scenes))(*[s.handle.value for s in scenes])
        arr = (_lib.Batch * len(batches))()
        for i, b in enumerate(batches):
            arr[i].scene = b.scene
            arr[i].n = int(b.tmax.shape[0])
            arr[i].flags = _lib.RQ_ANYHIT if b.anyhit else _lib.RQ_CLOSEST
            arr[i].d_org = b.org.data_ptr()
            arr[i].d_dir = b.dir.data_ptr()
            arr[i].d_tmax = b.tmax.data_ptr()
            arr[i].d_t = self.t[i].data_ptr()
            arr[i].d_prim = self.prim[i].data_ptr()
            arr[i].d_u = self.u[i].data_ptr() if self.u[i] is not None else None
            arr[i].d_v = self.v[i].data_ptr() if self.v[i] is not None else None
        self._arr = arr
        self.total_rays = sum(int(b.tmax.shape[0]) for b in batches)
        self._plan = C.c_void_p()
        self.config = None
        self.make_plan(config)

    def _cfg(self, config):
        if config is None:
            return None
        c = _lib.BatchConfig()
        c.block_threads = config.get("block_threads", 128)
        c.blocks_per_sm = config.get("blocks_per_sm", 0)
        c.chunk_rays = config.get("chunk_rays", 128)
        c.refill_threshold = config.get("refill_threshold", 8)
        c.reg_stack = config.get("reg_stack", 0)
        c.node_layout = config.get("node_layout", 0)
        c.smem_entries = config.get("smem_entries", 0)
        return c

    def make_plan(self, config: dict | None = None) -> None:
        self.close()
        cfg = self._cfg(config)
        check(lib.rq_batch_plan_create(self._scene_arr, len(self.scenes), self._arr,
                                       len(self.batches), C.byref(cfg) if cfg else None,
                                       C.byref(self._plan)))
        got = _lib.BatchConfig()
        grid = C.c_int()
        n = C.c_longlong()
        check(lib.rq_batch_plan_info(self._plan, C.byref(got), C.byref(grid), C.byref(n)))
        self.config = got.as_dict()
        self.grid = grid.value

    def autotune(self, reps: int = 2, candidates: list[dict] | None = None) -> dict:
        best = _lib.BatchConfig()
        ms = C.c_float()
        cand = None
        if candidates:
            cand = (_lib.BatchConfig * len(candidates))(*[self._cfg(c) for c in candidates])
        check(lib.rq_batch_autotune(self._scene_arr, len(self.scenes), self._arr,
                                    len(self.batches), cand, len(candidates or []), reps,
                                    C.byref(best), C.byref(ms)))
        self.make_plan(best.as_dict())
        self.tuned_ms = ms.value
        return best.as_dict()

    def launch(self, stream: int = 0) -> None:
        check(lib.rq_batch_plan_launch(self._plan, C.c_void_p(stream or None)))

    def close(self) -> None:
        if self._plan:
            lib.rq_batch_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
