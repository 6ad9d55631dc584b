"""Benchmark of the ray-query path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload path_frame|small_frame]

Prints ONE JSON line (rank 0).  A step is one frame of the named workload:

  path_frame   (default) incoherent path tracing: 1280x720, 16 spp
               stratified jitter, diffuse bounces to depth 4 with cosine
               hemisphere sampling from per-path PCG32 streams, Russian
               roulette from depth 1 as KajiyaPathtracer does (survivors
               unscaled, as in the reference), one parallelogram area light sampled
               with a shadow ray at every bounce, over a 512x1024 fBm
               heightfield (1,048,576 triangles) plus 32 displaced level-4
               icospheres (163,840 triangles).  Rays per step = camera +
               bounce rays + shadow rays traced.
  small_frame  512x512, 1 spp primary + hard-shadow rays from one point
               light over a displaced level-6 icosphere (81,920 triangles)
               and a 2x2 ground grid of 20,000 triangles.
  coherent_frame
               1920x1080, 4 spp jittered primary + hard-shadow rays from two
               point lights over a two-level scene: a 1024x1024 fBm
               heightfield (2,097,152 triangles) plus 64 InstanceT copies of
               a displaced level-6 icosphere (81,920 triangles each).

value     Mrays/s with the scene and frame buffers resident in HBM, device
          time from CUDA events around each frame, L2 flushed (a 256 MiB
          write) before every timed frame; whole job = sum over ranks.
e2e       Same metric through the host-buffer call (rq_render_path /
          rq_render_whitted: parameters in, the image copied back to host
          memory every frame), host wall clock per frame.
roofline  The dominant kernel of the frame: algorithmic bytes (rays x
          (32 + 16|4 + 32 x box tests per ray + 48 x triangle tests per ray),
          test counts from the library's statistics mode on the same frame)
          over its CUDA-event time, against the measured HBM copy peak.
cpu_baseline / --impl reference
          The reference's own CPU renderer on the same scene and camera
          (KajiyaPathtracer or Raytracer, DynBVH, WaldTriangle, Lambertian,
          HardShadows; MANTA_SSE build compiled from the reference sources
          into oracle/_ref by oracle/ref.mk) on all host cores, on a bounded
          sample of the frame.

With --gpus N (torchrun) every rank renders the same frame on its own GPU:
the path has no exchange step, so ranks are independent replicas (weak
scaling); the only collectives are the timing barrier and the max-over-ranks
reduction.
"""
from __future__ import annotations

import argparse
import ctypes as C
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s primary+diffuse on 1 B200 vs plain GPU form & host CPU; p99 request ms"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def pinned(shape, dtype=np.float32):
    """A host array in pinned (page-locked) memory, where the end-to-end
    numbers read each step's result."""
    import torch
    t = torch.empty(shape, dtype={np.float32: torch.float32, np.int32: torch.int32}[dtype],
                    pin_memory=True)
    return t.numpy()


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_over_ranks(x: float, op: str = "max", device=None) -> float:
    """x reduced over the process group ("max" for step times, "sum" for
    rates); the value itself when no group is running."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(rays_per_step: int, steps: int, world: int, seconds: float) -> float:
    """Whole-job Mrays/s: every rank traces rays_per_step per step (weak
    scaling), over the slowest rank's time."""
    return rays_per_step * steps * world / seconds / 1e6


# ------------------------------------------------------------- workloads ---

class PathFrame:
    name = "path_frame"

    def __init__(self):
        from rfmanta_b200 import scenes
        self.sc = scenes.path_scene()

    def config(self):
        sc = self.sc
        return {"workload": self.name, "resolution": [sc.xres, sc.yres], "spp": sc.spp,
                "max_depth": sc.max_depth, "russian_roulette_from": sc.rr_depth,
                "triangles": int(sc.mesh.n_tris), "lights": "1 parallelogram area light",
                "triangle_kind": "wald", "tree": "gpu binned SAH",
                "l2": "flushed before every timed frame (256 MiB write)"}

    def setup(self, bvh, dev):
        import torch
        self.bvh = bvh
        self.params = bvh.path_params(self.sc, chunk_paths=self.sc.xres * self.sc.yres * self.sc.spp)
        npx = self.sc.xres * self.sc.yres
        self.rgb = torch.empty(npx * 3, device=dev)
        self.counts = torch.zeros(2, dtype=torch.int64, device=dev)
        self.n_events = 2 + 2 * self.sc.max_depth
        self.stage_names = []
        for d in range(self.sc.max_depth):
            self.stage_names += [f"path_extend_persistent_kernel[{d}]", f"path_shade_persistent_kernel[{d}]"]
        self.stage_names.append("path_resolve_kernel")
        # per frame: generate and resolve, and per bounce the ray count,
        # extension, shade and the three ordered-compaction kernels
        self.launches = 2 + 6 * self.sc.max_depth

    def frame(self, stream_ptr):
        self.bvh.render_path_device(self.params, self.rgb.data_ptr(), self.counts.data_ptr(),
                                    stream_ptr)

    def rays(self):
        c = self.counts.cpu().numpy()
        return int(c[0]), int(c[1])

    def host_frame(self):
        """One frame through the host-buffer call; returns bytes in/out."""
        from rfmanta_b200 import _lib
        sc = self.sc
        if not hasattr(self, "_host_rgb"):
            self._host_rgb = pinned((sc.xres * sc.yres, 3))
            self._host_counts = (C.c_uint64 * 2)()
        _lib.check(_lib.lib.rq_render_path(self.bvh.handle, C.byref(self.params),
                                           self._host_rgb.ctypes.data, self._host_counts))
        return C.sizeof(self.params), self._host_rgb.nbytes + 16

    def roofline_bytes(self, stats, rays):
        """Algorithmic bytes of the extend stage (all bounces) and of the
        fused shade stage (its shadow rays)."""
        ext, shadow = rays
        b_e, t_e = stats[0] / max(ext, 1), stats[1] / max(ext, 1)
        b_s, t_s = stats[2] / max(shadow, 1), stats[3] / max(shadow, 1)
        per_ray = {"extension_box_tests": round(b_e, 3), "extension_tri_tests": round(t_e, 3),
                   "shadow_box_tests": round(b_s, 3), "shadow_tri_tests": round(t_s, 3)}
        return (ext * (32 + 16 + 32 * b_e + 48 * t_e),
                shadow * (32 + 4 + 32 * b_s + 48 * t_s)), per_ray

    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per extension
    # ray of path_extend_persistent_kernel: one ncu capture of the four
    # launches (bounces 0-3) of one full-size frame of this workload
    # (1280x720x16, 26.5M extension rays), summed over the launches and
    # divided by their rays.
    DRAM_BYTES_PER_RAY = 65.7
    DRAM_BASIS = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the 4 "
                  "path_extend_persistent_kernel launches of one full-size frame (1.744 GB "
                  "over 26,534,621 extension rays = 65.7 B per ray) x extension rays per "
                  "launch (all bounces / depth)")

    def traffic(self, rays):
        ext, _ = rays
        per_launch = self.DRAM_BYTES_PER_RAY * ext / self.sc.max_depth
        return per_launch, self.DRAM_BASIS

    def launches_of(self, stage):
        return self.sc.max_depth

    # What bounds the extension kernel, from one `ncu --set full` capture of
    # bounce 0 at 640x360x4 spp (same scene): lanes active per warp
    # instruction, warps active vs the occupancy limit, issue-slot use,
    # L1/TEX and L2 throughput, long-scoreboard stalls per issued
    # instruction.
    LIMITER = {"limiter": "dependent-load latency and SIMT efficiency, not HBM bandwidth",
               "lanes_per_warp_instruction": 15.2, "warps_active_pct": 35.0,
               "warps_active_theoretical_pct": 56.0, "issue_active_pct": 52.0,
               "l1tex_throughput_pct": 40.5, "l2_throughput_pct": 6.2,
               "long_scoreboard_stalls_per_issue": 5.71,
               "profile": "profiles/path_extend_persistent_kernel_path_frame.md"}

    def limiter(self):
        return dict(self.LIMITER)

    def image_check(self):
        """The device frame (16 spp) against the reference's KajiyaPathtracer
        frames of the cpu_baseline sample (independent 16 spp frames of the
        same camera, scene and light), in expectation: per 16x16-pixel tile,
        the difference of the two estimates of the tile's mean radiance, in
        absolute terms and in standard errors (variance of a 16-spp pixel
        estimate measured across the reference's frames).  The device image
        itself equals the restatement bit for bit (maximum per-channel error
        0; tests/test_gpu_parity_full.py)."""
        if getattr(self, "ref_image", None) is None or not hasattr(self, "_host_rgb"):
            return None
        acc, acc2, n = self.ref_image
        sc = self.sc
        T = 16
        ty, tx = sc.yres // T, sc.xres // T

        def tiles(a):
            a = a.reshape(sc.yres, sc.xres, 3)[:ty * T, :tx * T]
            return a.reshape(ty, T, tx, T, 3).mean(axis=(1, 3))
        ref_mean = tiles(acc / n)
        # variance of one 16-spp pixel estimate, from the spread of each
        # pixel across the reference's n frames (unbiased), averaged over the
        # tile; the reference's tile mean averages T^2 n such estimates, the
        # device's T^2 (one frame)
        var = np.maximum(tiles(acc2 / n) - tiles((acc / n) ** 2), 0.0) * n / max(n - 1, 1)
        dev_mean = tiles(self._host_rgb.astype(np.float64))
        se = np.sqrt(var / (T * T * n) + var / (T * T))
        d = dev_mean - ref_mean
        # tiles without variance (background only) are compared exactly
        noisy = se > 0
        z = np.abs(d)[noisy] / se[noisy]
        return {"vs_restatement_max_abs_error": 0.0,
                "vs_reference_expectation": {
                    "tiles": int(ty * tx), "tile_pixels": T * T, "reference_spp": int(n),
                    "device_spp": int(sc.spp),
                    "max_abs_tile_mean_diff": [round(float(x), 5) for x in np.abs(d).max(axis=(0, 1))],
                    "mean_tile_radiance": [round(float(x), 5) for x in ref_mean.mean(axis=(0, 1))],
                    "max_abs_z": round(float(z.max()), 2) if z.size else None,
                    "frac_tiles_abs_z_gt_3": round(float((z > 3).mean()), 5) if z.size else None,
                    "zero_variance_tile_channels": int((~noisy).sum()),
                    "zero_variance_tile_channels_differing": int((d[~noisy] != 0).sum()),
                    "image_mean_z": [round(float(x), 2) for x in
                                     (d.mean(axis=(0, 1)) /
                                      np.maximum(np.sqrt((se ** 2).sum(axis=(0, 1))), 1e-30)
                                      * (ty * tx))]}}

    def group_stages(self, stage_ms):
        D = self.sc.max_depth
        ext = sum(stage_ms[2 * d] for d in range(D))
        shade = sum(stage_ms[2 * d + 1] for d in range(D))
        return ["path_extend_persistent_kernel", "path_shade_persistent_kernel"], [ext, shade]

    def cpu_reference(self, seconds_budget, threads):
        """Reference KajiyaPathtracer on a 1 spp sample of the same frame."""
        from dataclasses import replace
        from oracle.pyoracle import Reference
        sse = Reference.available(sse=True)
        ref = Reference(sse=sse)
        t0 = time.perf_counter()
        rs = ref.scene(self.sc.mesh, 0)  # Mesh + DynBVH::rebuild, one thread
        build_s = time.perf_counter() - t0
        frames, secs, rays = 0, 0.0, 0
        acc = np.zeros((self.sc.xres * self.sc.yres, 3), np.float64)
        acc2 = np.zeros_like(acc)
        while frames < 1 or secs < seconds_budget:
            # independent full frames (16 spp stratified jitter, the
            # harness's sampler seeded per frame), accumulated for the
            # expectation comparison with the device frame
            sample = replace(self.sc, seed=self.sc.seed + 1000 + frames)
            out = rs.render_path(sample, nthreads=threads)
            secs += out["seconds"]
            rays += out["rays"]
            frames += 1
            acc += out["rgb"]
            acc2 += out["rgb"].astype(np.float64) ** 2
        rs.close()
        self.ref_image = (acc, acc2, frames)
        text = (f"{frames} full frame(s) of {sample.xres}x{sample.yres} at {sample.spp} spp, "
                f"depth {sample.max_depth}, reference KajiyaPathtracer/DynBVH/"
                f"WaldTriangle/Lambertian/HardShadows/AreaLight "
                f"({'MANTA_SSE' if sse else 'scalar'} build), rays counted at DynBVH::intersect; "
                f"the reference's DynBVH::rebuild of the scene took {build_s:.2f} s")
        return rays / secs / 1e6, threads, text, secs


def scenes_camera_rays(sc):
    """Primary rays of a WhittedScene's pinhole camera in pixel order (row
    by row), as 3 x n origin and direction arrays (pixel centres; the
    library's own frame uses the reference's camera on the device)."""
    cam = sc.camera
    eye = np.asarray(cam.eye, np.float64)
    look = np.asarray(cam.lookat, np.float64) - eye
    up = np.asarray(cam.up, np.float64)
    w = look / np.linalg.norm(look)
    u = np.cross(w, up)
    u /= np.linalg.norm(u)
    v = np.cross(u, w)
    tu = np.tan(np.radians(cam.hfov) / 2)
    tv = np.tan(np.radians(cam.vfov) / 2)
    ys, xs = np.mgrid[0:sc.yres, 0:sc.xres]
    px = ((xs + 0.5) / sc.xres * 2 - 1).ravel() * tu
    py = ((ys + 0.5) / sc.yres * 2 - 1).ravel() * tv
    d = (w[:, None] + u[:, None] * px[None, :] + v[:, None] * py[None, :])
    d /= np.linalg.norm(d, axis=0)
    o = np.repeat(eye[:, None], d.shape[1], axis=1)
    return o.astype(np.float32), d.astype(np.float32)


class SmallFrame:
    name = "small_frame"

    def __init__(self):
        from rfmanta_b200 import scenes
        self.sc = scenes.small_frame_scene()

    def config(self):
        sc = self.sc
        return {"workload": self.name, "resolution": [sc.xres, sc.yres], "spp": 1,
                "triangles": int(sc.mesh.n_tris), "lights": len(sc.lights),
                "triangle_kind": "wald", "tree": "gpu binned SAH",
                "l2": "flushed before every timed frame (256 MiB write)"}

    def setup(self, bvh, dev):
        import torch
        self.bvh = bvh
        self.params = bvh.whitted_params(self.sc)
        npx = self.sc.xres * self.sc.yres
        self.rgb = torch.empty(npx * 3, device=dev)
        self.t = torch.empty(npx, device=dev)
        self.prim = torch.empty(npx, dtype=torch.int32, device=dev)
        self.nshadow = torch.zeros(1, dtype=torch.int64, device=dev)
        self.n_events = 2
        self.stage_names = ["whitted_fused_kernel"]
        self.launches = 1

    def frame(self, stream_ptr):
        self.bvh.render_whitted_device(self.params, self.rgb.data_ptr(), self.t.data_ptr(),
                                       self.prim.data_ptr(), self.nshadow.data_ptr(), stream_ptr)

    def rays(self):
        return self.sc.xres * self.sc.yres, int(self.nshadow.item())

    def host_frame(self):
        from rfmanta_b200 import _lib
        npx = self.sc.xres * self.sc.yres
        if not hasattr(self, "_h"):
            self._h = (pinned((npx, 3)), pinned(npx), pinned(npx, np.int32), C.c_uint64())
        rgb, t, p, ns = self._h
        _lib.check(_lib.lib.rq_render_whitted(self.bvh.handle, C.byref(self.params),
                                              rgb.ctypes.data, t.ctypes.data, p.ctypes.data,
                                              C.byref(ns)))
        return C.sizeof(self.params) + 24 * len(self.sc.lights), npx * 20 + 8

    def roofline_bytes(self, stats, rays):
        prim, shadow = rays
        b_p, t_p = stats[0] / max(prim, 1), stats[1] / max(prim, 1)
        b_s, t_s = stats[2] / max(shadow, 1), stats[3] / max(shadow, 1)
        per_ray = {"primary_box_tests": round(b_p, 3), "primary_tri_tests": round(t_p, 3),
                   "shadow_box_tests": round(b_s, 3), "shadow_tri_tests": round(t_s, 3)}
        # one kernel traces both kinds of ray
        return (prim * (32 + 16 + 32 * b_p + 48 * t_p) +
                shadow * (32 + 4 + 32 * b_s + 48 * t_s),), per_ray

    # DRAM bytes per pixel of whitted_fused_kernel, from one ncu capture of
    # this workload at full size (262,144 pixels: 4.84 MB read, 0.02 MB
    # written).
    DRAM_BYTES_PER_PIXEL = 18.6

    def traffic(self, rays):
        prim, _ = rays
        return self.DRAM_BYTES_PER_PIXEL * prim, (
            f"ncu DRAM bytes of one whitted_fused_kernel launch at full size "
            f"({self.DRAM_BYTES_PER_PIXEL} B per pixel)")

    def group_stages(self, stage_ms):
        return self.stage_names, [stage_ms[0]]

    def cpu_reference(self, seconds_budget, threads):
        from oracle.pyoracle import Reference
        sse = Reference.available(sse=True)
        ref = Reference(sse=sse)
        t0 = time.perf_counter()
        rs = ref.scene(self.sc.mesh, 0)  # Mesh + DynBVH::rebuild, one thread
        build_s = time.perf_counter() - t0
        frames, secs, rays = 0, 0.0, 0
        while frames < 1 or secs < seconds_budget:
            out = rs.render(self.sc, nthreads=threads, want_ids=False)
            secs += out["seconds"]
            rays += self.sc.xres * self.sc.yres + out["shadow_rays"]
            frames += 1
        rs.close()
        text = (f"{frames} full {self.sc.xres}x{self.sc.yres} frame(s), reference Raytracer/"
                f"DynBVH/WaldTriangle/Lambertian/HardShadows "
                f"({'MANTA_SSE' if sse else 'scalar'} build); the reference's DynBVH::rebuild "
                f"of the scene took {build_s:.2f} s")
        return rays / secs / 1e6, threads, text, secs

    def extra(self, dev):
        """Per-packet latency of the frame's own camera rays: 64-ray packets
        (one image row segment each, as Manta's workers make them) traced
        one at a time from host arrays through rq_trace (a launch and a
        synchronise per packet) and through the resident packet channel;
        the channel's own records split its round trip into device time and
        the rest (PCIe signalling and host wait)."""
        from rfmanta_b200 import _lib
        sc = self.sc
        cam = scenes_camera_rays(sc)
        o, d = cam
        npk = 512
        pk = [(np.ascontiguousarray(o[:, 64 * k:64 * k + 64]),
               np.ascontiguousarray(d[:, 64 * k:64 * k + 64]),
               np.full(64, 1e19, np.float32)) for k in range(npk)]
        t = np.zeros(64, np.float32)
        pr = np.zeros(64, np.int32)
        ch = C.c_void_p()
        _lib.check(_lib.lib.rq_channel_create(self.bvh.handle, 16, 1024, C.byref(ch)))

        def run(fn, h):
            for oo, dd, tm in pk[:32]:  # warm-up
                _lib.check(fn(h, 64, oo.ctypes.data, dd.ctypes.data, tm.ctypes.data,
                              _lib.RQ_CLOSEST, t.ctypes.data, pr.ctypes.data, None, None))
            t0 = time.perf_counter()
            for oo, dd, tm in pk:
                _lib.check(fn(h, 64, oo.ctypes.data, dd.ctypes.data, tm.ctypes.data,
                              _lib.RQ_CLOSEST, t.ctypes.data, pr.ctypes.data, None, None))
            return (time.perf_counter() - t0) / npk * 1e6

        per_call = run(_lib.lib.rq_trace, self.bvh.handle)
        resident = run(_lib.lib.rq_channel_trace, ch)
        p_, r_, n_ = C.c_longlong(), C.c_longlong(), C.c_longlong()
        dev_us, rt_us = C.c_double(), C.c_double()
        _lib.check(_lib.lib.rq_channel_stats(ch, C.byref(p_), C.byref(r_), C.byref(n_),
                                             C.byref(dev_us), C.byref(rt_us)))
        _lib.lib.rq_channel_destroy(ch)
        return {"packet_latency_us": {
            "packet": "64 camera rays of one image row, closest hit, one caller thread",
            "per_call_rq_trace": round(per_call, 2),
            "resident_channel": round(resident, 2),
            "resident_channel_device": round(dev_us.value, 2),
            "resident_channel_round_trip": round(rt_us.value, 2)}}

    def dropin_rates(self, threads, seconds=1.5):
        """The reference's own renderer on the host cores with the drop-in
        swapped in: Manta's Raytracer + Lambertian + HardShadows (the
        reference's classes compiled here in the MANTA_SSE build the CPU
        baseline uses, oracle/_ref/libmanta_dropin_sse.so) tracing every
        64-ray packet through
        GpuDynBVH, one packet per call, on `threads` render workers.  Packets
        reach the device per call (rq_trace: a launch and a synchronise
        each), through the resident packet channel (rq_channel_*), and
        through the channel with GpuHardShadows for the shadow rays.
        Mrays/s of whole frames (primary + shadow rays)."""
        from oracle.pyoracle import DROPIN_SO, DROPIN_SSE_SO, Reference
        path = DROPIN_SSE_SO if os.path.exists(DROPIN_SSE_SO) else DROPIN_SO
        if not os.path.exists(path):
            return None
        ref = Reference(path=path)
        rs = ref.scene(self.sc.mesh, 0)
        rs.use_gpu(0, 0)  # the drop-in's own GPU-built tree
        npx = self.sc.xres * self.sc.yres
        build = "MANTA_SSE" if path == DROPIN_SSE_SO else "scalar"
        out = {"threads": threads,
               "frame": f"{self.sc.xres}x{self.sc.yres}, 1 spp, Raytracer/Lambertian/"
                        f"HardShadows of the reference ({build} build) over GpuDynBVH"}
        def rate(workers):
            rs.render(self.sc, nthreads=workers, want_ids=False)  # warm-up
            secs, rays, frames = 0.0, 0, 0
            while frames < 2 or secs < seconds:
                o = rs.render(self.sc, nthreads=workers, want_ids=False)
                secs += o["seconds"]
                rays += npx + o["shadow_rays"]
                frames += 1
            return round(rays / secs / 1e6, 2)

        for name, mode, gpu_shadows in (("per_call", 0, False), ("resident", 2, False),
                                        ("resident_gpu_shadows", 2, True)):
            rs.gpu_options(mode=mode, gpu_shadows=gpu_shadows)
            out[f"{name}_mrays"] = rate(threads)
        # more render workers than cores: a worker waiting on its packet
        # yields the core to one that shades
        rs.gpu_options(mode=2, gpu_shadows=True)
        out["resident_gpu_shadows_workers_mrays"] = {str(w): rate(w) for w in
                                                     (2 * threads, 4 * threads, 8 * threads)}
        rs.gpu_options(mode=0)
        rs.close()
        return out


class CoherentFrame:
    """1920x1080, 4 spp jittered primary + hard-shadow rays from two point
    lights over a two-level scene: a 1024x1024 fBm heightfield (2,097,152
    triangles, nested DynBVH) plus 64 InstanceT copies of a displaced level-6
    icosphere (81,920 triangles each)."""

    name = "coherent_frame"

    def __init__(self):
        from rfmanta_b200 import scenes
        self.sc = scenes.coherent_scene()

    def config(self):
        sc = self.sc
        return {"workload": self.name, "resolution": [sc.xres, sc.yres], "spp": sc.spp,
                "triangles_instanced": sc.n_tris,
                "triangles_stored": int(sum(m.n_tris for m in sc.inner)),
                "instances": int(np.count_nonzero(sc.kind == 0)),
                "lights": len(sc.lights), "triangle_kind": "wald",
                "tree": "gpu binned SAH (inner and top level)",
                "l2": "flushed before every timed frame (256 MiB write)"}

    def build(self, dev):
        from rfmanta_b200.dynbvh import GpuDynBVH, InstancedBVH
        self.inner = []
        self.build_s = 0.0
        for m in self.sc.inner:
            b = GpuDynBVH(tri_kind=0, device=dev.index or 0)
            b.setGroup(m)
            b.rebuild()
            self.build_s += b.build_seconds()
            self.inner.append(b)
        top = InstancedBVH(self.inner, self.sc.inst_scene, self.sc.translation, self.sc.kind)
        top.rebuild()
        self.build_s += top.build_seconds()
        return top

    def setup(self, bvh, dev):
        import torch
        self.bvh = bvh
        self.params = bvh.frame_params(self.sc, self.sc.materials)
        npx = self.sc.xres * self.sc.yres
        self.rgb = torch.empty(npx * 3, device=dev)
        self.nshadow = torch.zeros(1, dtype=torch.int64, device=dev)
        self.n_events = 4
        self.stage_names = ["frame_primary_kernel", "frame_shade_kernel", "frame_resolve_kernel"]
        self.launches = 3

    def frame(self, stream_ptr):
        self.bvh.render_frame_device(self.params, self.rgb.data_ptr(), self.nshadow.data_ptr(),
                                     stream_ptr)

    def rays(self):
        return self.sc.xres * self.sc.yres * self.sc.spp, int(self.nshadow.item())

    def host_frame(self):
        from rfmanta_b200 import _lib
        npx = self.sc.xres * self.sc.yres
        if not hasattr(self, "_h"):
            self._h = (pinned((npx, 3)), C.c_uint64())
        rgb, ns = self._h
        _lib.check(_lib.lib.rq_render_frame(self.bvh.handle, C.byref(self.params),
                                            rgb.ctypes.data, C.byref(ns)))
        return C.sizeof(self.params) + 24 * len(self.sc.lights), rgb.nbytes + 8

    def roofline_bytes(self, stats, rays):
        prim, shadow = rays
        b_p, t_p = stats[0] / max(prim, 1), stats[1] / max(prim, 1)
        b_s, t_s = stats[2] / max(shadow, 1), stats[3] / max(shadow, 1)
        per_ray = {"primary_box_tests": round(b_p, 3), "primary_tri_tests": round(t_p, 3),
                   "shadow_box_tests": round(b_s, 3), "shadow_tri_tests": round(t_s, 3)}
        return (prim * (32 + 16 + 32 * b_p + 48 * t_p),
                shadow * (32 + 4 + 32 * b_s + 48 * t_s),
                12 * prim + 12 * (prim // self.sc.spp)), per_ray

    # DRAM bytes per primary ray of frame_primary_kernel, from one ncu
    # capture of this workload at 960x540 x 1 spp (518,400 rays, same scene).
    DRAM_BYTES_PER_RAY = 127.7

    def traffic(self, rays):
        prim, _ = rays
        return self.DRAM_BYTES_PER_RAY * prim, ("ncu DRAM bytes per primary ray at 960x540x1 "
                                                "(127.7 B) x primary rays of the launch")

    def group_stages(self, stage_ms):
        return self.stage_names, [stage_ms[0], stage_ms[1], stage_ms[2]]

    def cpu_reference(self, seconds_budget, threads):
        """Reference Raytracer over the reference's own two-level DynBVH
        (InstanceT objects + the nested heightfield DynBVH) on every 16th
        image row of the frame's samples."""
        from oracle.pyoracle import Reference, Restatement
        sse = Reference.available(sse=True)
        sc = self.sc
        if not hasattr(self, "_ref"):  # the reference's trees, built once
            ref = Reference(sse=sse)
            inner = [ref.scene(m, 0) for m in sc.inner]
            self._ref = (ref, inner, ref.instanced(inner, sc.inst_scene, sc.translation,
                                                   sc.kind))
        top = self._ref[2]
        rs = Restatement()
        per_row = sc.xres * sc.spp
        rows = list(range(0, sc.yres, 16))
        cs = [rs.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed,
                               items=(y * per_row, (y + 1) * per_row)) for y in rows]
        px = np.concatenate([c[0] for c in cs])
        py = np.concatenate([c[1] for c in cs])
        passes, secs, rays = 0, 0.0, 0
        while passes < 1 or secs < seconds_budget:
            t0 = time.perf_counter()
            out = top.render_coords(sc, px, py, nthreads=threads)
            secs += time.perf_counter() - t0
            rays += px.size + out["shadow_rays"]
            passes += 1
        text = (f"{passes} pass(es) over every 16th row of the {sc.xres}x{sc.yres}x{sc.spp} "
                f"frame ({len(rows)} rows, {px.size} samples), reference Raytracer over a "
                f"top-level DynBVH of InstanceT + nested DynBVH objects, WaldTriangle/"
                f"Lambertian/HardShadows ({'MANTA_SSE' if sse else 'scalar'} build)")
        return rays / secs / 1e6, threads, text, secs


class BatchedQueriesWL:
    """64 ray batches (log-uniform 1k-4M rays, 50% any hit with tmax uniform
    in [0.1, diag], 50% closest hit) over 8 resident scenes of 10,240 to
    5,120,000 triangles, one persistent launch replayed from a CUDA graph
    with the autotuned configuration."""

    name = "batched_queries"

    def __init__(self, scale=1.0, plan_config=None):
        from rfmanta_b200 import scenes
        self.specs = scenes.query_batches(scale=scale)
        self.meshes = [scenes.query_scene(i) for i in range(8)]
        self.sc = None
        self.scale = scale
        self.plan_config = plan_config  # None: autotuned

    def config(self):
        return {"workload": self.name, "scenes": [int(m.n_tris) for m in self.meshes],
                "batches": len(self.specs), "rays": int(sum(n for _, n, _ in self.specs)),
                "batch_scale": self.scale,
                "anyhit_batches": int(sum(a for _, _, a in self.specs)),
                "triangle_kind": "wald", "tree": "gpu binned SAH",
                "l2": "flushed before every timed step (256 MiB write); inputs exceed L2"}

    def build(self, dev):
        from rfmanta_b200.dynbvh import GpuDynBVH
        self.bvhs = []
        self.build_s = 0.0
        for m in self.meshes:
            b = GpuDynBVH(tri_kind=0, device=dev.index or 0)
            b.setGroup(m)
            b.rebuild()
            self.build_s += b.build_seconds()
            self.bvhs.append(b)
        return self.bvhs[0]

    def setup(self, bvh, dev):
        from rfmanta_b200 import scenes
        from rfmanta_b200.batch import BatchedQueries, QueryBatch
        self.batches = []
        for k, (si, n, anyhit) in enumerate(self.specs):
            lo, hi = self.meshes[si].bounds()
            o, d, tm = scenes.query_rays_torch(n, lo, hi, anyhit, seed=1000 + k, device=dev)
            self.batches.append(QueryBatch(si, o, d, tm, anyhit))
        self.bq = BatchedQueries(self.bvhs, self.batches, self.plan_config)
        self.tuned = self.bq.autotune(reps=3) if self.plan_config is None else self.bq.config
        self.n_events = 0
        self.launches = 1
        self.total = self.bq.total_rays

    def frame(self, stream_ptr):
        self.bq.launch(stream_ptr)

    def rays(self):
        return (self.total,)

    def set_stats(self, ptr):
        # stats are collected by a plan created while scene 0 counts
        from rfmanta_b200.batch import BatchedQueries
        self.bvhs[0].set_stats(ptr)
        if ptr:
            self._stats_bq = BatchedQueries(self.bvhs, self.batches, self.tuned)
        else:
            self._stats_bq.close()

    def stats_frame(self, stream_ptr):
        self._stats_bq.launch(stream_ptr)

    def host_frame(self):
        """Host arrays in pinned memory: rays copied in, the plan replayed,
        t and triangle ids copied back."""
        import torch
        if not hasattr(self, "_pinned"):
            self._pinned = [(b.org.cpu().pin_memory(), b.dir.cpu().pin_memory(),
                             b.tmax.cpu().pin_memory(),
                             torch.empty(b.tmax.shape[0], pin_memory=True),
                             torch.empty(b.tmax.shape[0], dtype=torch.int32, pin_memory=True))
                            for b in self.batches]
        for b, (o, d, tm, _, _) in zip(self.batches, self._pinned):
            b.org.copy_(o, non_blocking=True)
            b.dir.copy_(d, non_blocking=True)
            b.tmax.copy_(tm, non_blocking=True)
        self.bq.launch(torch.cuda.current_stream().cuda_stream)
        for i, (_, _, _, t, p) in enumerate(self._pinned):
            t.copy_(self.bq.t[i], non_blocking=True)
            p.copy_(self.bq.prim[i], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return 28 * self.total, 8 * self.total

    def roofline_bytes(self, stats, rays):
        n = rays[0]
        b, t = stats[0] / max(n, 1), stats[1] / max(n, 1)
        # 32 B ray in; 8 B (t, id) out for closest, 4 for any hit: 6 on average
        return (n * (32 + 6 + 32 * b + 48 * t),), {"box_tests": round(b, 3),
                                                    "tri_tests": round(t, 3)}

    def group_stages(self, frame_ms):
        return ["batch_kernel"], [frame_ms]

    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per ray of
    # batch_kernel: one ncu capture of the same 64 batches scaled by 1/4
    # (7,080,009 rays; 1,275.7 MB read, 75.7 MB written) with the autotuned
    # kind of configuration (split stack, 8 shared entries), scaled to a
    # full launch by its rays (the batches and scenes are the same, so the
    # re-read pattern per ray carries over).
    DRAM_BYTES_PER_RAY = 190.9

    # What bounds batch_kernel, from one `ncu --set full` capture at 1/4 of
    # the batch sizes (split stack, 8 shared entries, 48 registers).
    LIMITER = {"limiter": "dependent-load latency and SIMT efficiency on uniformly random rays, "
                          "not HBM bandwidth",
               "lanes_per_warp_instruction": 8.67, "warps_active_pct": 55.2,
               "warps_active_theoretical_pct": 62.5, "issue_active_pct": 61.5,
               "long_scoreboard_stalls_per_issue": 7.88, "l1_hit_pct": 60.3,
               "l2_hit_pct": 61.4}

    def limiter(self):
        return dict(self.LIMITER)

    def traffic(self, rays):
        n = rays[0]
        return self.DRAM_BYTES_PER_RAY * n, (
            f"ncu DRAM bytes per ray of batch_kernel at 1/4 of the batch sizes "
            f"({self.DRAM_BYTES_PER_RAY} B) x rays of the launch")

    def legs(self, dev, reps=5):
        """Device time of the batched plan and of the plain per-call form
        (one rq_trace_device launch per batch, in batch order) over the same
        rays, each rep after the same 256 MiB L2 flush; Mrays/s of each."""
        import torch
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream

        def plain():
            for i, b in enumerate(self.batches):
                n = int(b.tmax.shape[0])
                self.bvhs[b.scene].intersect_device(n, b.org.data_ptr(), b.dir.data_ptr(),
                                                    b.tmax.data_ptr(), b.anyhit,
                                                    self.bq.t[i].data_ptr(),
                                                    self.bq.prim[i].data_ptr(), stream=st)

        out = {}
        for name, fn in (("batched", lambda: self.bq.launch(st)), ("plain", plain)):
            fn()
            ms = []
            for k in range(reps):
                flush.fill_(k & 0xff)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fn()
                e1.record()
                torch.cuda.synchronize(dev)
                ms.append(e0.elapsed_time(e1))
            out[name] = self.total / (sum(ms) / reps * 1e-3) / 1e6
        return out

    def extra(self, dev):
        """The plain per-call GPU form (one rq_trace_device launch per batch,
        timed like the batched leg) and Manta's per-packet form (rq_trace on
        64-ray host packets)."""
        legs = self.legs(dev)
        return {"plain_gpu_per_batch_mrays": round(legs["plain"], 1),
                "batched_vs_plain": round(legs["batched"] / legs["plain"], 3),
                "per_packet_calls_mrays": round(self.per_packet_rate(), 2),
                "per_packet_calls": "64-ray rq_trace calls (host arrays) from 16 host threads "
                                    "at once, rays of the first batch",
                "autotuned": self.tuned, "build_ms_total": round(self.build_s * 1e3, 1)}

    def per_packet_rate(self, threads=16, packets_per_thread=400):
        """The per-call drop-in form as Manta's workers use it: every host
        thread traces 64-ray packets from host arrays with rq_trace, one
        call at a time; Mrays/s over all threads (ctypes releases the
        interpreter lock during each call)."""
        from rfmanta_b200 import _lib
        b = self.batches[0]
        n = 64 * packets_per_thread
        o = np.ascontiguousarray(b.org[:, :n].cpu().numpy())
        d = np.ascontiguousarray(b.dir[:, :n].cpu().numpy())
        tm = np.ascontiguousarray(b.tmax[:n].cpu().numpy())
        npk = o.shape[1] // 64
        pk = [(np.ascontiguousarray(o[:, 64 * k:64 * k + 64]),
               np.ascontiguousarray(d[:, 64 * k:64 * k + 64]),
               np.ascontiguousarray(tm[64 * k:64 * k + 64])) for k in range(npk)]
        h = self.bvhs[b.scene].handle
        flags = _lib.RQ_ANYHIT if b.anyhit else _lib.RQ_CLOSEST

        def work():
            t = np.zeros(64, np.float32)
            p = np.zeros(64, np.int32)
            for po, pd, pt in pk:
                _lib.lib.rq_trace(h, 64, po.ctypes.data, pd.ctypes.data, pt.ctypes.data, flags,
                                  t.ctypes.data, p.ctypes.data, None, None)

        th = [threading.Thread(target=work) for _ in range(threads)]
        t0 = time.perf_counter()
        for x in th:
            x.start()
        for x in th:
            x.join()
        return threads * npk * 64 / (time.perf_counter() - t0) / 1e6

    def cpu_reference(self, seconds_budget, threads):
        """Reference DynBVH::intersect (64-ray packets, all host threads) on
        the batches of the five scenes up to 1M triangles, 300k rays of each
        batch at most."""
        import numpy as np
        from oracle.pyoracle import Reference
        from rfmanta_b200 import scenes
        sse = Reference.available(sse=True)
        ref = Reference(sse=sse)
        cache, secs, rays, used = {}, 0.0, 0, 0
        for k, (si, n, anyhit) in enumerate(self.specs):
            if si > 4:
                continue
            if si not in cache:
                cache[si] = ref.scene(self.meshes[si], 0)
            lo, hi = self.meshes[si].bounds()
            m = min(n, 300000)
            o, d, tm, _ = scenes.random_rays(m, lo, hi, seed=k, anyhit_fraction=1.0 if anyhit else 0.0)
            if not anyhit:
                tm = np.full(m, 1e19, np.float32)
            out = cache[si].intersect_mt(o, d, tm, anyhit=anyhit, nthreads=threads)
            secs += out["seconds"]
            rays += m
            used += 1
            if secs > seconds_budget > 0:
                break
        for r in cache.values():
            r.close()
        text = (f"{used} batches ({rays} rays, at most 300k per batch) on the scenes of up to "
                f"983,040 triangles, reference DynBVH::intersect on 64-ray packets "
                f"({'MANTA_SSE' if sse else 'scalar'} build)")
        return rays / secs / 1e6, threads, text, secs


class ServingWL(BatchedQueriesWL):
    """Poisson stream (mean 200 requests/s, seeded) of render requests over
    the 8 resident scenes: resolution from {256^2, 512^2, 1280x720,
    1920x1080}, spp from {1, 4, 16}, bounce depth from {0, 2, 4}; served by
    the continuous-batching engine (16Mi-path wavefront steps, 256Ki-pixel
    chunks, images admitted against an HBM budget; the request loop runs in
    the library, rq_server_run_stream).  A step is one stream of `requests`
    requests (at least 5 streams); value = rays traced / wall time from the
    first submit to the last completion, over all streams."""

    name = "serving"
    requests = 64

    def config(self):
        return {"workload": self.name, "scenes": [int(m.n_tris) for m in self.meshes],
                "requests_per_step": self.requests, "arrival_rate_per_s": 200,
                "resolutions": ["256x256", "512x512", "1280x720", "1920x1080"],
                "spp": [1, 4, 16], "bounces": [0, 2, 4], "path_capacity": SERVE_CAPACITY,
                "chunk_pixels": SERVE_CHUNK, "triangle_kind": "wald", "tree": "gpu binned SAH"}

    def run_custom(self, args, dev):
        self.build(dev)
        r = measure_serving(self.meshes, self.bvhs, [100 + k for k in range(max(args.steps, 5))],
                            self.requests, saturated=True, e2e=True)
        return {"value": r["served_mrays"], "ms_per_step": r["wall_ms_per_stream"],
                "e2e": r["e2e_mrays"], "h2d": r["h2d_bytes"], "d2h": r["d2h_bytes"],
                "rays_per_step": r["rays_per_stream"],
                "extra": {k: v for k, v in r.items()
                          if k not in ("served_mrays", "e2e_mrays", "h2d_bytes", "d2h_bytes",
                                       "rays_per_stream", "wall_ms_per_stream")}}

    def cpu_reference(self, seconds_budget, threads):
        """Reference KajiyaPathtracer on 256x256 requests of the scenes up to
        983,040 triangles (1 spp, depth 3)."""
        from oracle.pyoracle import Reference
        from rfmanta_b200 import scenes
        from rfmanta_b200.serve import request_for_scene
        sse = Reference.available(sse=True)
        ref = Reference(sse=sse)
        secs, rays, used = 0.0, 0, 0
        for si in range(5):
            r = request_for_scene(si, self.meshes[si], 256, 256, 1, 3, seed=si)
            ps = scenes.PathScene(self.meshes[si], scenes.Camera(r.eye, r.lookat, r.up, r.hfov,
                                                                 r.vfov),
                                  scenes.AreaLightSpec(r.light_anchor, r.light_v1, r.light_v2,
                                                       r.light_color),
                                  r.background, 256, 256, 1, 3, 2, r.seed)
            rs = ref.scene(self.meshes[si], 0)
            o = rs.render_path(ps, nthreads=threads)
            rs.close()
            secs += o["seconds"]
            rays += o["rays"]
            used += 1
        text = (f"{used} requests of 256x256, 1 spp, depth 3 on the scenes of up to 983,040 "
                f"triangles, reference KajiyaPathtracer ({'MANTA_SSE' if sse else 'scalar'} build)")
        return rays / secs / 1e6, threads, text, secs


SERVE_CAPACITY = 1 << 24   # paths per step
SERVE_CHUNK = 262144       # whole pixels per chunk


def measure_serving(meshes, bvhs, seeds, requests, saturated=False, e2e=False):
    """The continuous-batching server and serial plain calls on the same
    seeded Poisson streams (200 requests/s): served throughput = rays traced
    / (first submit to last completion), summed over the streams; the median
    stream too; p50/p99 request latency.  Serial FIFO: each request rendered
    alone by rq_render_path (service time on the host clock), replayed in
    arrival order against the same arrival times."""
    from rfmanta_b200 import scenes
    from rfmanta_b200.serve import RenderServer, poisson_stream
    srv = RenderServer(bvhs, path_capacity=SERVE_CAPACITY, chunk_pixels=SERVE_CHUNK,
                       hbm_budget_bytes=24 << 30)
    srv.run_stream(poisson_stream(meshes, 8, 200.0, seed=3))
    rays, wall, lat, queue, per = 0, 0.0, [], [], []
    for sd in seeds:
        b0 = srv.stats()
        out = srv.run_stream(poisson_stream(meshes, requests, 200.0, seed=sd))
        st = srv.stats()
        r = (st["rays"] - b0["rays"]) + (st["shadow_rays"] - b0["shadow_rays"])
        rays += r
        wall += out["wall_s"]
        per.append(r / out["wall_s"] / 1e6)
        lat += [v["latency"] for v in out["info"].values()]
        queue += [v["queue"] for v in out["info"].values()]
    res = {}
    if e2e:
        b0 = srv.stats()
        stream = poisson_stream(meshes, requests, 200.0, seed=seeds[0])
        out = srv.run_stream(stream, keep_images=True)
        st = srv.stats()
        er = (st["rays"] - b0["rays"]) + (st["shadow_rays"] - b0["shadow_rays"])
        res.update(e2e_mrays=rays_or(er) / out["wall_s"] / 1e6, h2d_bytes=200 * requests,
                   d2h_bytes=sum(q.xres * q.yres * 12 for _, q in stream))
    srv.close()
    if saturated:
        srv = RenderServer(bvhs, path_capacity=SERVE_CAPACITY, chunk_pixels=SERVE_CHUNK,
                           hbm_budget_bytes=24 << 30)
        stream = poisson_stream(meshes, requests, 200.0, seed=seeds[0])
        b0 = srv.stats()
        sat = srv.run_stream([(0.0, q) for _, q in stream])
        st = srv.stats()
        res["saturated_served_mrays"] = round(
            ((st["rays"] - b0["rays"]) + (st["shadow_rays"] - b0["shadow_rays"]))
            / sat["wall_s"] / 1e6, 1)
        srv.close()
    serial_rays, serial_lat, serial_wall, serial_service, serial_per = 0, [], 0.0, 0.0, []
    for sd in seeds:
        sk = poisson_stream(meshes, requests, 200.0, seed=sd)
        service, srays = [], 0
        for _, q in sk:
            ps = scenes.PathScene(meshes[q.scene],
                                  scenes.Camera(q.eye, q.lookat, q.up, q.hfov, q.vfov),
                                  scenes.AreaLightSpec(q.light_anchor, q.light_v1, q.light_v2,
                                                       q.light_color),
                                  q.background, q.xres, q.yres, q.spp, q.max_depth,
                                  q.rr_depth, q.seed)
            t0 = time.perf_counter()
            o = bvhs[q.scene].render_path(ps)
            service.append(time.perf_counter() - t0)
            srays += o["rays"] + o["shadow_rays"]
        finish = 0.0
        for (arr, _), sv in zip(sk, service):
            finish = max(finish, arr) + sv
            serial_lat.append(finish - arr)
        serial_wall += finish - sk[0][0]
        serial_service += sum(service)
        serial_rays += srays
        serial_per.append(srays / (finish - sk[0][0]) / 1e6)
    lat_ms = np.array(lat) * 1e3
    serial_ms = np.array(serial_lat) * 1e3
    res.update({
        "served_mrays": rays / wall / 1e6,
        "served_median_stream_mrays": round(float(np.median(per)), 1),
        "p50_ms": round(float(np.percentile(lat_ms, 50)), 2),
        "p99_ms": round(float(np.percentile(lat_ms, 99)), 2),
        "mean_admission_wait_ms": round(float(np.mean(queue) * 1e3), 2),
        "serial_fifo_mrays": round(serial_rays / serial_wall / 1e6, 1),
        "serial_fifo_median_stream_mrays": round(float(np.median(serial_per)), 1),
        "serial_fifo_p50_ms": round(float(np.percentile(serial_ms, 50)), 2),
        "serial_fifo_p99_ms": round(float(np.percentile(serial_ms, 99)), 2),
        "saturated_serial_mrays": round(serial_rays / serial_service / 1e6, 1),
        "streams": len(seeds), "requests_per_stream": requests,
        "rays_per_stream": rays // max(len(seeds), 1),
        "wall_ms_per_stream": wall / max(len(seeds), 1) * 1e3,
        "path_capacity": SERVE_CAPACITY, "chunk_pixels": SERVE_CHUNK,
    })
    return res


def system_forms(dev, streams=3):
    """The two system forms beside the plain per-call form, measured in the
    same run: the batched-query plan against plain per-batch calls (same
    rays, same L2 flush), and the server against serial plain calls over
    seeded Poisson streams."""
    wl = BatchedQueriesWL()
    wl.build(dev)
    wl.setup(None, dev)
    legs = wl.legs(dev)
    out = {"batched_mrays": round(legs["batched"], 1),
           "plain_per_batch_mrays": round(legs["plain"], 1),
           "batched_vs_plain": round(legs["batched"] / legs["plain"], 3),
           "per_packet_calls_mrays": round(wl.per_packet_rate(), 2),
           "batched_autotuned": wl.tuned,
           "batched_workload": "64 batches, 1k-4M rays, 8 scenes of 10k-5.12M triangles, "
                               "50% any hit; L2 flushed (256 MiB) before every rep of both legs"}
    wl.bq.close()
    sv = measure_serving(wl.meshes, wl.bvhs, [100 + k for k in range(streams)], 64,
                         saturated=True)
    out.update({"served_mrays": round(sv["served_mrays"], 1),
                "served_p50_ms": sv["p50_ms"], "served_p99_ms": sv["p99_ms"],
                "serial_fifo_mrays": sv["serial_fifo_mrays"],
                "serial_fifo_p50_ms": sv["serial_fifo_p50_ms"],
                "serial_fifo_p99_ms": sv["serial_fifo_p99_ms"],
                "saturated_served_mrays": sv["saturated_served_mrays"],
                "saturated_serial_mrays": sv["saturated_serial_mrays"],
                "served_vs_serial_saturated": round(sv["saturated_served_mrays"] /
                                                    sv["saturated_serial_mrays"], 3),
                "serving_workload": f"{streams} Poisson streams x 64 requests at 200/s over the "
                                    f"8 scenes, {SERVE_CAPACITY} paths per step, "
                                    f"{SERVE_CHUNK}-pixel chunks"})
    for b in wl.bvhs:
        b.close()
    return out


def quick_rate(wl, dev, steps=5, warmup=3):
    """Device and end-to-end Mrays/s of one frame workload, timed like the
    main line (L2 flushed before every timed frame, CUDA events on the
    launching stream; e2e through the host-buffer call), for the compact
    record of the other workloads on the default line."""
    import torch
    from rfmanta_b200.dynbvh import GpuDynBVH
    if hasattr(wl, "build"):
        bvh = wl.build(dev)
    else:
        bvh = GpuDynBVH(tri_kind=0, device=dev.index or 0)
        bvh.setGroup(wl.sc.mesh)
        bvh.rebuild()
    wl.setup(bvh, dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        wl.frame(stream.cuda_stream)
    torch.cuda.synchronize(dev)
    rays = sum(wl.rays())
    ms = 0.0
    for k in range(steps):
        flush.fill_(k & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        wl.frame(stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize(dev)
        ms += a.elapsed_time(b)
    e2e = 0.0
    for k in range(warmup + steps):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        wl.host_frame()
        if k >= warmup:
            e2e += time.perf_counter() - t0
    del flush
    return {"value": round(rays * steps / (ms * 1e-3) / 1e6, 1),
            "e2e": round(rays * steps / e2e / 1e6, 1),
            "ms_per_step": round(ms / steps, 4), "rays_per_step": int(rays),
            "steps": steps, "warmup": warmup}


def make_workload(args):
    if args.workload == "batched_queries":
        wl = BatchedQueriesWL(args.batch_scale,
                              json.loads(args.batch_config) if args.batch_config else None)
    else:
        if args.batch_scale != 1.0 or args.batch_config:
            raise SystemExit("--batch-scale/--batch-config apply to batched_queries")
        wl = WORKLOADS[args.workload]()
    sc = getattr(wl, "sc", None)
    if (args.res or args.spp) and sc is None:
        raise SystemExit(f"--res/--spp apply to frame workloads, not {args.workload}")
    if args.res:
        w, h = (int(x) for x in args.res.lower().split("x"))
        sc.xres, sc.yres = w, h
    if args.spp:
        sc.spp = args.spp
    return wl


def rays_or(x):
    return max(int(x), 1)


class AnimatedFrame(SmallFrame):
    """The 512x512 Whitted frame of a moving mesh: every step first moves
    the vertices (a periodic 8-frame wave, the positions resident on the
    device) and updates the tree as DynBVH::update does (refit, leaf
    re-splits, tree rotations), then renders."""
    name = "animated_frame"
    PERIOD = 8

    def __init__(self):
        super().__init__()
        from rfmanta_b200 import scenes
        self.v0 = self.sc.mesh.vertices.copy()
        self.poses = [scenes.wave_vertices(self.v0, k, self.PERIOD) for k in range(self.PERIOD)]
        self.k = 0

    def config(self):
        c = super().config()
        c.update({"workload": self.name,
                  "update": "DynBVH::update with tree rotations and leaf re-splits every frame",
                  "animation": f"periodic wave, {self.PERIOD} poses, amplitude 0.01",
                  "vertices": int(self.v0.shape[0])})
        return c

    def setup(self, bvh, dev):
        import torch
        super().setup(bvh, dev)
        # (3 floats per vertex, row-major: the library reads a plain array)
        self.dev_poses = [torch.from_numpy(np.ascontiguousarray(v)).to(dev).contiguous()
                          for v in self.poses]
        self.host_poses = [torch.from_numpy(np.ascontiguousarray(v)).pin_memory()
                           for v in self.poses]
        self.sc.mesh.vertices = self.poses[0]
        bvh.update()
        # kernels per step: 1 for the frame; the update's state reset, object
        # boxes, leaf boxes, re-splits, 2 scan kernels, relocation, next-free
        # advance, rotations, parents, 1 + 9 pointer-jumping rounds, records
        # and the triangle records
        self.launches = 1 + 21

    def frame(self, stream_ptr):
        k = self.k % self.PERIOD
        self.k += 1
        self.sc.mesh.vertices = self.poses[k]
        self.bvh.update_device(self.dev_poses[k].data_ptr(), rotate=True, stream=stream_ptr)
        super().frame(stream_ptr)

    def host_frame(self):
        from rfmanta_b200 import _lib
        k = self.k % self.PERIOD
        self.k += 1
        v = self.host_poses[k]
        self.sc.mesh.vertices = self.poses[k]
        _lib.check(_lib.lib.rq_scene_update_vertices_ex(self.bvh.handle, C.c_void_p(v.data_ptr()),
                                                        v.shape[0], _lib.RQ_UPDATE_ROTATE))
        h2d, d2h = super().host_frame()
        return h2d + v.numel() * 4, d2h

    def cpu_reference(self, seconds_budget, threads):
        from oracle.pyoracle import Reference
        sse = Reference.available(sse=True)
        ref = Reference(sse=sse)
        rs = ref.scene(self.sc.mesh, 0)
        frames, secs, rays, upd = 0, 0.0, 0, 0.0
        while frames < 2 or secs < seconds_budget:
            v = self.poses[frames % self.PERIOD]
            t0 = time.perf_counter()
            rs.update_vertices(v)
            du = time.perf_counter() - t0
            self.sc.mesh.vertices = v
            out = rs.render(self.sc, nthreads=threads, want_ids=False)
            secs += du + out["seconds"]
            upd += du
            rays += self.sc.xres * self.sc.yres + out["shadow_rays"]
            frames += 1
        rs.close()
        self.sc.mesh.vertices = self.v0
        text = (f"{frames} full {self.sc.xres}x{self.sc.yres} animated frame(s): reference "
                f"DynBVH::update(0, 1) (single-threaded, {1e3 * upd / frames:.1f} ms per frame) "
                f"then Raytracer/DynBVH/WaldTriangle/Lambertian/HardShadows on {threads} "
                f"thread(s) ({'MANTA_SSE' if sse else 'scalar'} build)")
        return rays / secs / 1e6, threads, text, secs


WORKLOADS = {"path_frame": PathFrame, "small_frame": SmallFrame,
             "animated_frame": AnimatedFrame,
             "coherent_frame": CoherentFrame,
             "batched_queries": BatchedQueriesWL, "serving": ServingWL}


# ----------------------------------------------------------------- runs ----

def run_ours(args):
    import torch
    import torch.distributed as dist
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=datetime.timedelta(seconds=120))
    from rfmanta_b200.dynbvh import GpuDynBVH
    wl = make_workload(args)
    dev = torch.device("cuda", local)
    if hasattr(wl, "run_custom"):
        return run_custom(args, wl, dev, world, rank)
    if hasattr(wl, "build"):
        bvh = wl.build(dev)
        build_s = wl.build_s
    else:
        bvh = GpuDynBVH(tri_kind=0, device=local)
        bvh.setGroup(wl.sc.mesh)
        bvh.rebuild()
        build_s = bvh.build_seconds()
    wl.setup(bvh, dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    # statistics frame (untimed): box / triangle tests per ray
    stats = torch.zeros(4, dtype=torch.int64, device=dev)
    if hasattr(wl, "stats_frame"):
        wl.set_stats(stats.data_ptr())
        wl.stats_frame(sptr)
        torch.cuda.synchronize(dev)
        wl.set_stats(0)
    else:
        bvh.set_stats(stats.data_ptr())
        wl.frame(sptr)
        torch.cuda.synchronize(dev)
        bvh.set_stats(0)
    st = stats.cpu().numpy().astype(np.float64)
    rays = wl.rays()
    rays_per_step = sum(rays)

    for _ in range(args.warmup):
        wl.frame(sptr)
    torch.cuda.synchronize(dev)

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(wl.n_events)]
    for e in ev:  # torch creates the CUDA event on first record
        e.record(stream)
    pairs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
             for _ in range(args.steps)]
    stage = np.zeros((args.steps, max(wl.n_events - 1, 1)))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        if wl.n_events:
            bvh.set_stage_events(ev)
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            pairs[k][0].record(stream)
            wl.frame(sptr)
            pairs[k][1].record(stream)
            torch.cuda.synchronize(dev)
            for j in range(wl.n_events - 1):
                stage[k, j] = ev[j].elapsed_time(ev[j + 1])
            if not wl.n_events:
                stage[k, 0] = pairs[k][0].elapsed_time(pairs[k][1])
        if wl.n_events:
            bvh.set_stage_events([])
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    total_ms = reduce_over_ranks(sum(a.elapsed_time(b) for a, b in pairs), "max", dev)
    value = job_rate(rays_per_step, args.steps, world, total_ms * 1e-3)

    # end to end through the host-buffer public call
    e2e = []
    bin_ = bout = 0
    for k in range(args.warmup + args.steps):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        bin_, bout = wl.host_frame()
        t1 = time.perf_counter()
        if k >= args.warmup:
            e2e.append(t1 - t0)
    e2e_value = job_rate(rays_per_step, args.steps, world,
                         reduce_over_ranks(sum(e2e), "max", dev))

    # roofline of the dominant kernel: measured DRAM bytes per launch over its
    # CUDA-event launch time against the measured HBM copy peak; beside it
    # the cache-inclusive algorithmic bytes (every node and triangle record a
    # ray reads, L1/L2 hits included), which is why that figure can exceed
    # the HBM peak
    hbm, peak_kind = _peaks()
    mean_stage = stage.mean(axis=0)
    names, kms = wl.group_stages(mean_stage if wl.n_events else float(mean_stage[0]))
    alg, per_ray = wl.roofline_bytes(st, rays)
    dom = int(np.argmax(kms))
    launches = wl.launches_of(dom) if hasattr(wl, "launches_of") else 1
    launch_ms = kms[dom] / launches
    alg_gbs = alg[dom] / (kms[dom] * 1e-3) / 1e9
    traffic, traffic_basis = (wl.traffic(rays) if hasattr(wl, "traffic") and dom == 0
                              else (None, None))
    if traffic is not None:
        achieved, basis = traffic / (launch_ms * 1e-3) / 1e9, "dram"
    else:
        achieved, basis = alg_gbs, "algorithmic (cache-inclusive)"
    forms = None
    others = None
    if rank == 0 and world == 1 and args.system_forms and wl.name == "path_frame":
        forms = system_forms(dev)
        # the other frame workloads, compactly, so one run records all of them
        others = {}
        for cls in (SmallFrame, CoherentFrame, AnimatedFrame):
            w = cls()
            others[w.name] = quick_rate(w, dev)
            del w

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generators)",
            "config": dict(wl.config(), parallelism=f"replicas x{world}",
                           rays_per_step=rays_per_step, rays_split=list(rays),
                           build_ms=round(build_s * 1e3, 2),
                           **(wl.extra(dev) if hasattr(wl, "extra") else {})),
            "clocks": clk.summary(),
            "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(bin_), "d2h_bytes_per_step": int(bout)},
            "gpu_launches": wl.launches * args.steps,
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": round(achieved, 1),
                         "achieved_basis": basis,
                         "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4),
                         "traffic": None if traffic is None else int(traffic),
                         "traffic_basis": traffic_basis,
                         "launch_ms": round(launch_ms, 4),
                         "algorithmic_cache_inclusive": {
                             "achieved": round(alg_gbs, 1),
                             "frac_of_hbm_peak": round(alg_gbs / hbm, 4),
                             "bytes_per_launch": int(alg[dom] / launches),
                             "basis": "32 B per box test + 48 B per triangle test + ray in/out, "
                                      "counted at every visit (L1/L2 hits included)"},
                         **(wl.limiter() if hasattr(wl, "limiter") else {}),
                         "kernel_ms_per_step": {n: round(v, 4) for n, v in zip(names, kms)},
                         "per_ray": per_ray},
        }
        if forms:
            line["system_forms"] = forms
        if others:
            line["other_workloads"] = others
        if not args.no_cpu_baseline and world == 1:  # the host baseline: rank 0 at N=1
            v, threads, text, _ = wl.cpu_reference(args.cpu_seconds, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": round(v, 3), "unit": "Mrays/s", "cores": threads,
                                    "kind": "reference", "sample": text}
            if hasattr(wl, "image_check"):
                line["image_error"] = wl.image_check()
            if wl.name in ("path_frame", "small_frame"):
                # the per-packet drop-in form under the reference's own
                # renderer (512x512 small frame scene), beside the baseline
                line["manta_dropin"] = (wl if wl.name == "small_frame"
                                        else SmallFrame()).dropin_rates(threads)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_custom(args, wl, dev, world, rank):
    """Workloads that drive their own loop (serving): wall-clock rates."""
    import torch
    import torch.distributed as dist
    with ClockSampler(dev.index or 0) as clk:
        r = wl.run_custom(args, dev)
    value = reduce_over_ranks(r["value"], "sum", dev)
    e2e = reduce_over_ranks(r["e2e"], "sum", dev)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(r["ms_per_step"], 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generators and request stream)",
            "config": dict(wl.config(), parallelism=f"replicas x{world}",
                           rays_per_step=r["rays_per_step"], **r["extra"]),
            "clocks": clk.summary(),
            "e2e": {"value": round(e2e, 2), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(r["h2d"]), "d2h_bytes_per_step": int(r["d2h"])},
            "gpu_launches": None,
            "roofline": None,
        }
        if not args.no_cpu_baseline and world == 1:  # the host baseline: rank 0 at N=1
            v, threads, text, _ = wl.cpu_reference(args.cpu_seconds, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": round(v, 3), "unit": "Mrays/s", "cores": threads,
                                    "kind": "reference", "sample": text}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def reference_config(cfg):
    """The workload's config as the reference arm runs it: the reference
    builds its own trees (DynBVH::rebuild, exact SAH sweep) and runs on the
    host cores, where no L2 flush applies."""
    cfg = dict(cfg)
    for k in ("tree",):
        if k in cfg:
            cfg[k] = "reference DynBVH::rebuild (exact SAH sweep), host CPU"
    for k in ("l2", "path_capacity", "chunk_pixels"):
        cfg.pop(k, None)
    cfg["l2"] = "not applicable (host CPU)"
    cfg["scheduling"] = ("the reference's Raytracer / KajiyaPathtracer / DynBVH::intersect on "
                         "64-ray packets, rows handed to host threads by the harness "
                         "(not RTRT's WorkQueue)")
    return cfg


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    from oracle.pyoracle import Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libmanta_ref.so was not built (needs the reference sources)"}))
        return
    wl = make_workload(args)
    threads = os.cpu_count() or 1
    per_step = []
    text = ""
    for k in range(args.warmup + args.steps):
        v, threads, text, secs = wl.cpu_reference(0.0, threads)
        if k >= args.warmup:
            per_step.append((v, secs))
    value = statistics.median([p[0] for p in per_step])
    ms = statistics.median([p[1] for p in per_step]) * 1e3
    print(json.dumps({
        "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene generators)", "impl": "reference",
        "config": reference_config(wl.config()),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads,
                         "kind": "reference", "sample": f"one sample per step: {text}"},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="path_frame", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-system-forms", dest="system_forms", action="store_false",
                    help="skip the batched / served comparison in the path_frame line")
    ap.add_argument("--res", default=None,
                    help="WxH override of a frame workload's resolution (small ncu cases)")
    ap.add_argument("--spp", type=int, default=None,
                    help="samples per pixel override of a frame workload")
    ap.add_argument("--batch-scale", type=float, default=1.0,
                    help="batched_queries: batch sizes scaled by this factor (small ncu cases)")
    ap.add_argument("--batch-config", default=None,
                    help="batched_queries: a fixed plan configuration (JSON) instead of the "
                         "autotuner's")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
