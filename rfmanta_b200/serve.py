"""Continuous-batching render server (rq_server_* in the C ABI).

``RenderServer`` wraps the native engine; ``run_stream`` drives it with a
timed arrival stream: requests are submitted when their arrival time comes,
the engine is stepped whenever it has work, finished requests are collected
and their latency (submit to completion observed on the host) recorded."""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, lib
from .dynbvh import fill_environment


@dataclass
class RenderRequest:
    scene: int
    eye: tuple
    lookat: tuple
    up: tuple
    hfov: float
    vfov: float
    xres: int
    yres: int
    spp: int
    max_depth: int
    rr_depth: int
    seed: int
    light_anchor: tuple
    light_v1: tuple
    light_v2: tuple
    light_color: tuple
    background: tuple
    materials: np.ndarray = field(default_factory=lambda: np.full((1, 3), 0.7, np.float32))
    ambient: tuple = (0.0, 0.0, 0.0)
    environment: object = None  # scenes.Environment, None = constant forms

    def to_c(self) -> _lib.ServeRequest:
        q = _lib.ServeRequest()
        q.scene = self.scene
        q.eye[:], q.lookat[:], q.up[:] = self.eye, self.lookat, self.up
        q.hfov, q.vfov = self.hfov, self.vfov
        q.xres, q.yres, q.spp = self.xres, self.yres, self.spp
        q.max_depth, q.rr_depth, q.seed = self.max_depth, self.rr_depth, self.seed
        q.light_anchor[:], q.light_v1[:], q.light_v2[:] = (self.light_anchor, self.light_v1,
                                                           self.light_v2)
        q.light_color[:], q.background[:] = self.light_color, self.background
        q.ambient[:] = self.ambient
        fill_environment(q.environment, self.environment)
        m = np.ascontiguousarray(self.materials, np.float32)
        q.n_materials = m.shape[0]
        q.material_rgb = m.ctypes.data
        q._keep = m
        return q

    @property
    def rays_upper(self) -> int:
        return self.xres * self.yres * self.spp * self.max_depth * 2


class RenderServer:
    def __init__(self, scenes, path_capacity: int = 1 << 22, chunk_pixels: int = 16384,
                 hbm_budget_bytes: int = 8 << 30):
        self.scenes = scenes
        arr = (C.c_void_p * len(scenes))(*[s.handle.value for s in scenes])
        self._h = C.c_void_p()
        check(lib.rq_server_create(arr, len(scenes), path_capacity, chunk_pixels,
                                   hbm_budget_bytes, C.byref(self._h)))

    def submit(self, req: RenderRequest) -> int:
        rid = C.c_int()
        q = req.to_c()
        check(lib.rq_server_submit(self._h, C.byref(q), C.byref(rid)))
        return rid.value

    def submit_query(self, scene: int, org, dir, tmax, anyhit: bool = False) -> int:
        """A ray-query request: host arrays (3, n), (3, n), (n,) float32,
        copied on submit; traced by the server's steps beside the renders."""
        o = np.ascontiguousarray(org, np.float32)
        d = np.ascontiguousarray(dir, np.float32)
        tm = np.ascontiguousarray(tmax, np.float32)
        q = _lib.ServeQuery(scene, int(tm.shape[0]), _lib.RQ_ANYHIT if anyhit else _lib.RQ_CLOSEST,
                            o.ctypes.data, d.ctypes.data, tm.ctypes.data)
        rid = C.c_int()
        check(lib.rq_server_submit_query(self._h, C.byref(q), C.byref(rid)))
        return rid.value

    def query_result(self, rid: int, n: int):
        """(t, triangle id, latency s, admission wait s) of a finished query."""
        t = np.empty(n, np.float32)
        prim = np.empty(n, np.int32)
        lat, qs = C.c_double(), C.c_double()
        check(lib.rq_server_query_result(self._h, rid, t.ctypes.data, prim.ctypes.data,
                                         C.byref(lat), C.byref(qs)))
        return t, prim, lat.value, qs.value

    def step(self) -> int:
        n = C.c_int()
        check(lib.rq_server_step(self._h, C.byref(n)))
        return n.value

    def poll(self) -> list[int]:
        ids = (C.c_int * 1024)()
        n = C.c_int()
        check(lib.rq_server_poll(self._h, ids, 1024, C.byref(n)))
        return list(ids[: n.value])

    def result(self, rid: int, xres: int, yres: int, copy: bool = True):
        rgb = np.empty((xres * yres, 3), np.float32) if copy else None
        lat, qs = C.c_double(), C.c_double()
        check(lib.rq_server_result(self._h, rid, rgb.ctypes.data if copy else None,
                                   C.byref(lat), C.byref(qs)))
        return rgb, lat.value, qs.value

    def release(self, rid: int) -> None:
        check(lib.rq_server_release(self._h, rid))

    def stats(self) -> dict:
        counts = (C.c_uint64 * 2)()
        steps, pend, act = C.c_longlong(), C.c_int(), C.c_int()
        used = C.c_size_t()
        check(lib.rq_server_stats(self._h, counts, C.byref(steps), C.byref(pend), C.byref(act),
                                  C.byref(used)))
        return dict(rays=int(counts[0]), shadow_rays=int(counts[1]), steps=steps.value,
                    pending=pend.value, active=act.value, bytes_in_use=used.value)

    def close(self) -> None:
        if self._h:
            lib.rq_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_stream(self, stream: list[tuple[float, RenderRequest]], keep_images: bool = False,
                   timeout_s: float = 600.0) -> dict:
        """Submits each request at its arrival time (seconds from start),
        steps until all are done (the loop runs in the library,
        rq_server_run_stream).  Returns per-request latencies and admission
        waits (s), the wall time from the first submit to the last
        completion and, optionally, the images."""
        n = len(stream)
        reqs = (_lib.ServeRequest * max(n, 1))()
        keep = []
        for i, (_, r) in enumerate(stream):
            q = r.to_c()
            keep.append(q._keep)
            reqs[i] = q
        arr = np.ascontiguousarray([a for a, _ in stream], np.float64)
        lat = np.zeros(n, np.float64)
        qs = np.zeros(n, np.float64)
        imgs = None
        ptrs = None
        if keep_images:
            imgs = [np.empty((r.xres * r.yres, 3), np.float32) for _, r in stream]
            ptrs = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in imgs])
        wall = C.c_double()
        check(lib.rq_server_run_stream(self._h, reqs, arr.ctypes.data, n, ptrs,
                                       lat.ctypes.data, qs.ctypes.data, C.byref(wall),
                                       float(timeout_s)))
        info = {i: dict(latency=float(lat[i]), queue=float(qs[i]),
                        image=imgs[i] if imgs else None) for i in range(n)}
        return dict(info=info, wall_s=wall.value)

    def set_profile(self, on: bool = True) -> None:
        check(lib.rq_server_set_profile(self._h, int(on)))

    def profile(self) -> list[dict]:
        """Finished steps' records since the last call (profiling on)."""
        out = []
        buf = (_lib.ServerStepRecord * 4096)()
        while True:
            n = C.c_int()
            check(lib.rq_server_profile(self._h, buf, 4096, C.byref(n)))
            out += [buf[i].as_dict() for i in range(n.value)]
            if n.value < 4096:
                return out


def request_for_scene(scene_index: int, mesh, xres: int, yres: int, spp: int,
                      max_depth: int, seed: int) -> RenderRequest:
    """A camera looking at the scene from above and in front, a parallelogram
    light above it."""
    lo, hi = mesh.bounds()
    c = (lo + hi) / 2
    ext = float(np.max(hi - lo))
    eye = (float(c[0]), float(hi[1] + 0.6 * ext), float(c[2] + 1.2 * ext))
    vfov = float(2 * np.degrees(np.arctan(np.tan(np.radians(30.0)) * yres / xres)))
    return RenderRequest(scene_index, eye, tuple(float(x) for x in c), (0.0, 1.0, 0.0), 60.0,
                         vfov, xres, yres, spp, max_depth, 2, seed,
                         (float(c[0] - 0.2 * ext), float(hi[1] + ext), float(c[2] - 0.2 * ext)),
                         (0.4 * ext, 0.0, 0.0), (0.0, 0.0, 0.4 * ext), (20.0, 19.0, 17.0),
                         (0.15, 0.2, 0.3), np.asarray(mesh.materials, np.float32))


def poisson_stream(meshes, n: int, rate: float = 200.0, seed: int = 11):
    """Seeded Poisson arrivals (mean `rate` per second) of render requests:
    scene uniform over `meshes`, resolution from {256^2, 512^2, 1280x720,
    1920x1080}, spp from {1, 4, 16}, bounce depth from {0, 2, 4}."""
    rng = np.random.default_rng(seed)
    res = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        si = int(rng.integers(0, len(meshes)))
        xr, yr = res[int(rng.integers(0, 4))]
        spp = int(rng.choice([1, 4, 16]))
        bounces = int(rng.choice([0, 2, 4]))
        out.append((t, request_for_scene(si, meshes[si], xr, yr, spp, bounces + 1,
                                         seed=1000 + i)))
    return out
