"""Benchmark of the ray-query path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload small_frame]

Prints ONE JSON line (rank 0).  A step is one frame of the named workload:

  small_frame  512x512, 1 spp pinhole primary rays + hard-shadow rays from
               one point light over a displaced level-6 icosphere (81,920
               triangles, seeded value noise, amplitude 0.05, frequency 4)
               and a 2x2 ground grid of 20,000 triangles; Lambertian
               shading; Wald triangles.  Rays per step = primary rays +
               shadow rays actually sent (the reference culls back-facing
               ones).

value     Mrays/s with the scene and frame buffers resident in HBM, device
          time from CUDA events around each frame, L2 flushed (a 256 MiB
          write) before every timed frame; whole job = sum over ranks.
e2e       Same metric through the host-buffer call rq_render_whitted (camera
          parameters in, RGB + primary t + triangle id copied back every
          frame), host wall clock per frame.
roofline  The dominant stage kernel: algorithmic bytes per launch
          (rays x (32 + 16|4 + 32 x box tests/ray + 48 x triangle tests/ray),
          test counts from the library's statistics mode on the same frame)
          over its CUDA-event duration, against the measured HBM copy peak.
cpu_baseline / --impl reference
          The reference's own CPU renderer for the same frame
          (Raytracer + DynBVH + WaldTriangle + Lambertian + HardShadows,
          MANTA_SSE build, compiled from the reference sources into
          oracle/_ref by oracle/ref.mk) on all host cores.

With --gpus N (torchrun) every rank renders the same frame on its own GPU:
the path has no exchange step, so the ranks are independent replicas
(weak scaling) and the only collectives are the timing barrier and the
max-over-ranks reduction.
"""
from __future__ import annotations

import argparse
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


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _workload(name):
    from rfmanta_b200 import scenes
    if name == "small_frame":
        return scenes.small_frame_scene()
    raise SystemExit(f"unknown workload {name}")


def _workload_config(name, sc):
    return {"workload": name, "resolution": [sc.xres, sc.yres], "spp": 1,
            "triangles": int(sc.mesh.n_tris), "lights": len(sc.lights),
            "triangle_kind": "wald", "tree": "gpu binned SAH",
            "l2": "flushed before every timed frame (256 MiB write)"}


def reference_frames(sc, seconds_budget: float, threads: int):
    """The reference's CPU renderer on the same frame, repeated within a
    time budget.  Returns (Mrays/s, frames, threads, kind, sample text)."""
    from oracle.pyoracle import Reference
    sse = Reference.available(sse=True)
    ref = Reference(sse=sse)
    rs = ref.scene(sc.mesh, 0)
    frames, secs, rays = 0, 0.0, 0
    while frames < 1 or secs < seconds_budget:
        out = rs.render(sc, nthreads=threads, want_ids=False)
        secs += out["seconds"]
        rays += sc.xres * sc.yres + out["shadow_rays"]
        frames += 1
    rs.close()
    kind = "reference"
    sample = (f"{frames} full {sc.xres}x{sc.yres} frame(s), reference Raytracer/DynBVH/"
              f"WaldTriangle/Lambertian/HardShadows ({'MANTA_SSE' if sse else 'scalar'} build)")
    return rays / secs / 1e6, frames, threads, kind, sample, secs


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    sc = _workload(args.workload)
    threads = os.cpu_count() or 1
    from oracle.pyoracle import Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libmanta_ref.so was not built (needs the reference sources)"}))
        return
    per_step = []
    for k in range(args.warmup + args.steps):
        v, frames, threads, kind, sample, secs = reference_frames(sc, 0.0, threads)
        if k >= args.warmup:
            per_step.append((v, secs))
    value = statistics.median([p[0] for p in per_step])
    ms = statistics.median([p[1] for p in per_step]) * 1e3
    print(json.dumps({
        "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene generators)", "impl": "reference",
        "config": _workload_config(args.workload, sc),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads,
                         "kind": kind, "sample": f"one frame per step: {sample}"},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import torch
    import torch.distributed as dist
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    from rfmanta_b200.dynbvh import GpuDynBVH
    sc = _workload(args.workload)
    bvh = GpuDynBVH(tri_kind=0, device=local)
    bvh.setGroup(sc.mesh)
    bvh.rebuild()
    build_s = bvh.build_seconds()
    params = bvh.whitted_params(sc)
    npx = sc.xres * sc.yres
    dev = torch.device("cuda", local)
    rgb = torch.empty(npx * 3, device=dev)
    tbuf = torch.empty(npx, device=dev)
    prim = torch.empty(npx, dtype=torch.int32, device=dev)
    nshadow = torch.zeros(1, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def frame():
        bvh.render_whitted_device(params, rgb.data_ptr(), tbuf.data_ptr(), prim.data_ptr(),
                                  nshadow.data_ptr(), sptr)

    # statistics frame (untimed): box / triangle tests per ray
    stats = torch.zeros(4, dtype=torch.int64, device=dev)
    bvh.set_stats(stats.data_ptr())
    frame()
    torch.cuda.synchronize(dev)
    bvh.set_stats(0)
    st = stats.cpu().numpy().astype(np.float64)
    n_shadow = int(nshadow.item())
    boxes_p, tris_p = st[0] / npx, st[1] / npx
    boxes_s, tris_s = st[2] / max(n_shadow, 1), st[3] / max(n_shadow, 1)

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize(dev)

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    for e in ev:  # torch creates the CUDA event on first record
        e.record(stream)
    pairs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
             for _ in range(args.steps)]
    stage = np.zeros((args.steps, 2))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        bvh.set_stage_events(ev)
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            pairs[k][0].record(stream)
            frame()
            pairs[k][1].record(stream)
            torch.cuda.synchronize(dev)
            stage[k, 0] = ev[0].elapsed_time(ev[1])
            stage[k, 1] = ev[1].elapsed_time(ev[2])
        bvh.set_stage_events([])
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    total_ms = sum(a.elapsed_time(b) for a, b in pairs)
    t_max = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    total_ms = float(t_max.item())
    rays_per_step = npx + n_shadow
    value = rays_per_step * args.steps * world / (total_ms * 1e-3) / 1e6

    # e2e through the host-buffer public call
    out_rgb = np.empty((npx, 3), np.float32)
    e2e_times = []
    from rfmanta_b200 import _lib
    import ctypes as C
    t_host = np.empty(npx, np.float32)
    p_host = np.empty(npx, np.int32)
    ns = C.c_uint64()
    for k in range(args.warmup + args.steps):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _lib.check(_lib.lib.rq_render_whitted(bvh.handle, C.byref(params),
                                              out_rgb.ctypes.data, t_host.ctypes.data,
                                              p_host.ctypes.data, C.byref(ns)))
        t1 = time.perf_counter()
        if k >= args.warmup:
            e2e_times.append(t1 - t0)
    e2e_secs = sum(e2e_times)
    e2e_t = torch.tensor([e2e_secs], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = rays_per_step * args.steps * world / float(e2e_t.item()) / 1e6

    # roofline of the dominant stage
    hbm, peak_kind = _peaks()
    mean_stage = stage.mean(axis=0)
    bytes_primary = npx * (32 + 16 + 32 * boxes_p + 48 * tris_p)
    bytes_shadow = n_shadow * (32 + 4 + 32 * boxes_s + 48 * tris_s)
    dom = int(np.argmax(mean_stage))
    alg = [bytes_primary, bytes_shadow][dom]
    achieved = alg / (mean_stage[dom] * 1e-3) / 1e9
    names = ["whitted_primary_kernel", "whitted_shade_kernel"]

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generators)",
            "config": dict(_workload_config(args.workload, sc), parallelism=f"replicas x{world}",
                           rays_per_step=rays_per_step, shadow_rays=n_shadow,
                           build_ms=round(build_s * 1e3, 2)),
            "clocks": clk.summary(),
            "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(C.sizeof(params) + 4 * 6 * len(sc.lights)),
                    "d2h_bytes_per_step": int(npx * 20 + 8)},
            "gpu_launches": 2 * args.steps,
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": round(achieved, 1),
                         "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4), "traffic": None,
                         "stage_ms": [round(x, 4) for x in mean_stage],
                         "per_ray": {"primary_box_tests": round(boxes_p, 3),
                                     "primary_tri_tests": round(tris_p, 3),
                                     "shadow_box_tests": round(boxes_s, 3),
                                     "shadow_tri_tests": round(tris_s, 3)}},
        }
        if not args.no_cpu_baseline:
            v, frames, threads, kind, sample, secs = reference_frames(sc, args.cpu_seconds,
                                                                      os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": round(v, 3), "unit": "Mrays/s", "cores": threads,
                                    "kind": kind, "sample": sample}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="small_frame")
    ap.add_argument("--cpu-seconds", type=float, default=5.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
