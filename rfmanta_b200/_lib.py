"""ctypes binding of the C ABI in include/rfmanta_b200.h.

The CUDA library must have been built (``python -m rfmanta_b200.build``);
there is no fallback path: importing this module without the library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librfmanta_b200.so")

RQ_OK = 0
RQ_ERR_NOTFOUND = 9
RQ_ERR_ARG = 1
RQ_ERR_CUDA = 2
RQ_ERR_OOM = 3
RQ_ERR_FORMAT = 4
RQ_ERR_STATE = 5
RQ_ERR_CAPACITY = 6
RQ_ERR_TIMEOUT = 7
RQ_ERR_NODEV = 8

RQ_TRI_WALD = 0
RQ_TRI_KS = 1
RQ_INST_TRANSLATE = 0
RQ_LAYOUT_DFS = 0
RQ_LAYOUT_BFS = 1
RQ_LAYOUT_BFS_TOP = 2
RQ_PATH_EXTEND = 2
RQ_PATH_SHADE = 3
RQ_MAT_LAMBERTIAN = 0
RQ_MAT_PHONG = 1
RQ_MAT_DIELECTRIC = 2
RQ_MAT_TRANSPARENT = 3
RQ_MAT_DEFAULT = 4
RQ_UPDATE_REFIT = 0
RQ_UPDATE_ROTATE = 1
RQ_INST_NESTED = 1
RQ_CLOSEST = 0
RQ_ANYHIT = 1

ERROR_NAMES = {
    RQ_ERR_ARG: "RQ_ERR_ARG", RQ_ERR_CUDA: "RQ_ERR_CUDA", RQ_ERR_OOM: "RQ_ERR_OOM",
    RQ_ERR_FORMAT: "RQ_ERR_FORMAT", RQ_ERR_STATE: "RQ_ERR_STATE",
    RQ_ERR_CAPACITY: "RQ_ERR_CAPACITY", RQ_ERR_TIMEOUT: "RQ_ERR_TIMEOUT",
    RQ_ERR_NODEV: "RQ_ERR_NODEV",
}


class RQError(RuntimeError):
    """A C-ABI call returned a non-zero status (the C++ shim maps these to
    Manta's InternalError)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


RQ_AMBIENT_CONSTANT, RQ_AMBIENT_EYE = 0, 1
RQ_BACKGROUND_CONSTANT, RQ_BACKGROUND_LINEAR = 0, 1


class EnvironmentParams(C.Structure):
    _fields_ = [("ambient_kind", C.c_int), ("background_kind", C.c_int),
                ("background_down", C.c_float * 3), ("background_up", C.c_float * 3)]


class WhittedParams(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("lookat", C.c_float * 3), ("up", C.c_float * 3),
                ("hfov", C.c_float), ("vfov", C.c_float), ("xres", C.c_int), ("yres", C.c_int),
                ("n_lights", C.c_int), ("lights", C.c_void_p), ("ambient", C.c_float * 3),
                ("background", C.c_float * 3), ("n_materials", C.c_int),
                ("material_rgb", C.c_void_p), ("environment", EnvironmentParams)]


class FrameParams(C.Structure):
    _fields_ = [("whitted", WhittedParams), ("spp", C.c_int), ("seed", C.c_uint64),
                ("material_specular", C.c_void_p), ("material_specpow", C.c_void_p),
                ("material_reflectivity", C.c_void_p), ("max_depth", C.c_int),
                ("importance_cutoff", C.c_float)]


class PathParams(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("lookat", C.c_float * 3), ("up", C.c_float * 3),
                ("hfov", C.c_float), ("vfov", C.c_float), ("xres", C.c_int), ("yres", C.c_int),
                ("spp", C.c_int), ("max_depth", C.c_int), ("rr_depth", C.c_int),
                ("seed", C.c_uint64), ("light_anchor", C.c_float * 3),
                ("light_v1", C.c_float * 3), ("light_v2", C.c_float * 3),
                ("light_color", C.c_float * 3), ("background", C.c_float * 3),
                ("ambient", C.c_float * 3), ("n_materials", C.c_int),
                ("material_rgb", C.c_void_p), ("chunk_paths", C.c_int),
                ("environment", EnvironmentParams)]


class Batch(C.Structure):
    _fields_ = [("scene", C.c_int), ("n", C.c_int), ("flags", C.c_int),
                ("d_org", C.c_void_p), ("d_dir", C.c_void_p), ("d_tmax", C.c_void_p),
                ("d_t", C.c_void_p), ("d_prim", C.c_void_p), ("d_u", C.c_void_p),
                ("d_v", C.c_void_p)]


class BatchConfig(C.Structure):
    _fields_ = [("block_threads", C.c_int), ("blocks_per_sm", C.c_int),
                ("chunk_rays", C.c_int), ("refill_threshold", C.c_int), ("reg_stack", C.c_int),
                ("node_layout", C.c_int), ("smem_entries", C.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServerStepRecord(C.Structure):
    _fields_ = [("requests", C.c_int), ("chunks", C.c_int), ("scenes", C.c_int),
                ("max_depth", C.c_int), ("paths", C.c_longlong), ("gpu_ms", C.c_float),
                ("t_enqueue_s", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServeQuery(C.Structure):
    _fields_ = [("scene", C.c_int), ("n", C.c_int), ("flags", C.c_int),
                ("org", C.c_void_p), ("dir", C.c_void_p), ("tmax", C.c_void_p)]


class ServeRequest(C.Structure):
    _fields_ = [("scene", C.c_int), ("eye", C.c_float * 3), ("lookat", C.c_float * 3),
                ("up", C.c_float * 3), ("hfov", C.c_float), ("vfov", C.c_float),
                ("xres", C.c_int), ("yres", C.c_int), ("spp", C.c_int), ("max_depth", C.c_int),
                ("rr_depth", C.c_int), ("seed", C.c_uint64), ("light_anchor", C.c_float * 3),
                ("light_v1", C.c_float * 3), ("light_v2", C.c_float * 3),
                ("light_color", C.c_float * 3), ("background", C.c_float * 3),
                ("ambient", C.c_float * 3), ("n_materials", C.c_int),
                ("material_rgb", C.c_void_p), ("environment", EnvironmentParams)]


class LaunchConfig(C.Structure):
    _fields_ = [("block_threads", C.c_int), ("blocks_per_sm", C.c_int),
                ("refill_threshold", C.c_int), ("persistent", C.c_int),
                ("reg_stack", C.c_int), ("node_layout", C.c_int)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m rfmanta_b200.build` "
            "(the ray-query path has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    vp, i, sz = C.c_void_p, C.c_int, C.c_size_t
    sig = {
        "rq_last_error": ([], C.c_char_p),
        "rq_version": ([], C.c_char_p),
        "rq_scene_create": ([vp, i, vp, i, vp, i, i, C.POINTER(vp)], i),
        "rq_scene_destroy": ([vp], i),
        "rq_scene_import_dynbvh": ([vp, vp, sz], i),
        "rq_scene_import_tree": ([vp, i, vp, vp, vp, vp, vp, vp], i),
        "rq_scene_build": ([vp, i], i),
        "rq_scene_sah_cost": ([vp, C.POINTER(C.c_double)], i),
        "rq_scene_info": ([vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(sz)], i),
        "rq_scene_export_dynbvh": ([vp, vp, C.POINTER(sz)], i),
        "rq_trace": ([vp, i, vp, vp, vp, i, vp, vp, vp, vp], i),
        "rq_trace_device": ([vp, i, vp, vp, vp, i, vp, vp, vp, vp, vp], i),
        "rq_set_launch_config": ([vp, i, C.POINTER(LaunchConfig)], i),
        "rq_get_launch_config": ([vp, i, C.POINTER(LaunchConfig)], i),
        "rq_camera_basis": ([vp, vp, vp, C.c_float, C.c_float, vp], i),
        "rq_render_whitted": ([vp, C.POINTER(WhittedParams), vp, vp, vp,
                               C.POINTER(C.c_uint64)], i),
        "rq_render_whitted_device": ([vp, C.POINTER(WhittedParams), vp, vp, vp, vp, vp], i),
        "rq_render_whitted_device_noalloc": ([vp, C.POINTER(WhittedParams), vp, vp, vp, vp,
                                              vp], i),
        "rq_set_stage_events": ([vp, vp, i], i),
        "rq_set_stats": ([vp, vp], i),
        "rq_render_path": ([vp, C.POINTER(PathParams), vp, vp], i),
        "rq_render_path_device": ([vp, C.POINTER(PathParams), vp, vp, vp], i),
        "rq_set_path_debug": ([vp, vp, vp, vp, C.c_int64], i),
        "rq_batch_plan_create": ([vp, i, vp, i, vp, C.POINTER(vp)], i),
        "rq_batch_plan_launch": ([vp, vp], i),
        "rq_batch_plan_info": ([vp, vp, C.POINTER(i), C.POINTER(C.c_longlong)], i),
        "rq_batch_plan_destroy": ([vp], i),
        "rq_batch_autotune": ([vp, i, vp, i, vp, i, i, vp, C.POINTER(C.c_float)], i),
        "rq_server_create": ([vp, i, C.c_longlong, i, sz, C.POINTER(vp)], i),
        "rq_server_submit": ([vp, C.POINTER(ServeRequest), C.POINTER(i)], i),
        "rq_server_step": ([vp, C.POINTER(i)], i),
        "rq_server_poll": ([vp, vp, i, C.POINTER(i)], i),
        "rq_server_result": ([vp, i, vp, C.POINTER(C.c_double), C.POINTER(C.c_double)], i),
        "rq_server_release": ([vp, i], i),
        "rq_server_stats": ([vp, vp, C.POINTER(C.c_longlong), C.POINTER(i), C.POINTER(i),
                             C.POINTER(sz)], i),
        "rq_server_destroy": ([vp], i),
        "rq_queue_create": ([vp, i, C.POINTER(vp)], i),
        "rq_queue_trace": ([vp, i, vp, vp, vp, i, vp, vp, vp, vp], i),
        "rq_queue_stats": ([vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                            C.POINTER(C.c_longlong)], i),
        "rq_queue_destroy": ([vp], i),
        "rq_channel_create": ([vp, i, i, C.POINTER(vp)], i),
        "rq_channel_trace": ([vp, i, vp, vp, vp, i, vp, vp, vp, vp], i),
        "rq_channel_set_timing": ([vp, C.c_double, C.c_double, C.c_double], i),
        "rq_channel_stats": ([vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                              C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                              C.POINTER(C.c_double)], i),
        "rq_channel_stop": ([vp], i),
        "rq_channel_destroy": ([vp], i),
        "rq_server_submit_query": ([vp, C.POINTER(ServeQuery), C.POINTER(i)], i),
        "rq_server_query_result": ([vp, i, vp, vp, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)], i),
        "rq_server_run_stream": ([vp, vp, vp, i, vp, vp, vp, C.POINTER(C.c_double), C.c_double],
                                 i),
        "rq_server_set_profile": ([vp, i], i),
        "rq_server_profile": ([vp, vp, i, C.POINTER(i)], i),
        "rq_scene_build_seconds": ([vp, C.POINTER(C.c_double)], i),
        "rq_scene_update_vertices": ([vp, vp, i], i),
        "rq_scene_update_vertices_ex": ([vp, vp, i, i], i),
        "rq_scene_update_vertices_device": ([vp, vp, i, i, vp], i),
        "rq_scene_update_state": ([vp, vp, i, vp], i),
        "rq_mesh_read_ply": ([C.c_char_p, vp, C.c_uint32, C.POINTER(vp)], i),
        "rq_mesh_info": ([vp, C.POINTER(i), C.POINTER(i)], i),
        "rq_mesh_copy": ([vp, vp, vp, vp], i),
        "rq_mesh_destroy": ([vp], i),
        "rq_mesh_read_obj": ([C.c_char_p, C.POINTER(vp)], i),
        "rq_mesh_material_count": ([vp, C.POINTER(i)], i),
        "rq_mesh_materials": ([vp] * 9, i),
        "rq_scene_create_instanced": ([vp, i, vp, vp, vp, i, C.POINTER(vp)], i),
        "rq_trace_device_ex": ([vp, i, vp, vp, vp, i, vp, vp, vp, vp, vp, vp], i),
        "rq_render_frame": ([vp, C.POINTER(FrameParams), vp, C.POINTER(C.c_uint64)], i),
        "rq_render_frame_device": ([vp, C.POINTER(FrameParams), vp, vp, vp], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


lib = _load()


def check(rc: int) -> None:
    if rc != RQ_OK:
        raise RQError(rc, lib.rq_last_error().decode(errors="replace"))


def declared_symbols(header: str | None = None) -> list[str]:
    """Entry points declared in include/rfmanta_b200.h."""
    import re
    header = header or os.path.join(os.path.dirname(HERE), "include", "rfmanta_b200.h")
    text = open(header).read()
    return sorted(set(re.findall(r"RQ_API\s+[\w\s\*]+?\b(rq_\w+)\s*\(", text)))
