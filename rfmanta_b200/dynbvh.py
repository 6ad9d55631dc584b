"""Python host mirror of the reference's ray-query interfaces.

``GpuDynBVH`` mirrors Manta's ``DynBVH : AccelerationStructure``
(Interface/AccelerationStructure.h:11-66, Model/Groups/DynBVH.h:151-224):
``setGroup``, ``groupDirty``, ``getGroup``, ``rebuild``, ``buildFromFile``,
``saveToFile``, ``computeBounds`` and ``intersect``.  ``RayBatch`` plays the
role of ``RayPacket`` (Interface/RayPacket.h:58-130) for any number of rays:
structure-of-arrays origins/directions, ``minT`` in and out, hit primitive,
scratchpad u/v and the ``AnyHit`` flag.  Every call goes through the C ABI
into the CUDA library; errors surface as ``RQError`` (the reference throws
``InternalError``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (RQ_ANYHIT, RQ_CLOSEST, RQ_TRI_KS, RQ_TRI_WALD, RQ_UPDATE_REFIT,
                   RQ_UPDATE_ROTATE, check, lib)
from .scenes import Mesh

T_EPSILON = np.float32(1.e-4)
MAXT = np.float32(1.e19)


def fill_environment(dst: "_lib.EnvironmentParams", env) -> None:
    """rq_environment from a scenes.Environment (None = the constant forms)."""
    if env is None:
        return
    dst.ambient_kind, dst.background_kind = env.kinds()
    dst.background_down[:] = env.background_down
    dst.background_up[:] = env.background_up


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class RayBatch:
    """Host-side ray batch (RayPacket semantics, any size).

    org, dir: (3, n) float32 SoA.  minT: (n,) float32, the query's upper
    bound on entry (RayPacket::resetHit) and the hit distance on exit.
    """

    AnyHit = RQ_ANYHIT

    def __init__(self, org, dir, minT=None, flags: int = 0):
        self.org = np.ascontiguousarray(org, np.float32).reshape(3, -1)
        self.dir = np.ascontiguousarray(dir, np.float32).reshape(3, -1)
        n = self.org.shape[1]
        self.minT = (np.full(n, MAXT, np.float32) if minT is None
                     else np.ascontiguousarray(minT, np.float32).copy())
        self.flags = flags
        self.hitPrim = np.full(n, -1, np.int32)
        self.u = np.zeros(n, np.float32)
        self.v = np.zeros(n, np.float32)

    def __len__(self):
        return self.org.shape[1]

    def getFlag(self, f: int) -> bool:
        return bool(self.flags & f)

    def setFlag(self, f: int) -> None:
        self.flags |= f

    def resetHits(self, maxt=MAXT) -> None:
        self.minT[:] = maxt
        self.hitPrim[:] = -1

    def wasHit(self) -> np.ndarray:
        return self.hitPrim >= 0


@dataclass
class SceneInfo:
    n_records: int
    n_leaves: int
    depth: int
    device_bytes: int


class GpuDynBVH:
    """AccelerationStructure over one triangle Mesh, on one GPU."""

    # how intersect() reaches the device (GpuDynBVH::setPacketMode in the
    # C++ drop-in): one rq_trace call each, or the resident packet channel
    PerCall, Resident = 0, 2

    def __init__(self, tri_kind: int = RQ_TRI_WALD, device: int = 0):
        self.tri_kind = tri_kind
        self.device = device
        self._h = C.c_void_p()
        self._ch = C.c_void_p()
        self._mode = self.PerCall
        self._group: Mesh | None = None
        self._dirty = False

    def setPacketMode(self, mode: int) -> None:
        """PerCall: every intersect() is an rq_trace call (one launch and one
        synchronise); Resident: calls of up to 1,024 rays go through a
        resident packet channel (rq_channel_*: a persistent kernel polls
        mapped host memory, no launch per call), made on first use."""
        if mode not in (self.PerCall, self.Resident):
            raise ValueError("PerCall or Resident")
        self._mode = mode
        if mode != self.Resident and self._ch:
            check(lib.rq_channel_stop(self._ch))

    # -- AccelerationStructure surface -------------------------------------
    def setGroup(self, group: Mesh) -> None:
        if group is not self._group:
            self._dirty = True
        self._group = group

    def getGroup(self) -> Mesh | None:
        return self._group

    def groupDirty(self) -> None:
        self._dirty = True

    def _upload(self) -> None:
        if self._group is None:
            raise _lib.RQError(_lib.RQ_ERR_STATE, "setGroup was not called")
        self.close()
        m = self._group
        v = np.ascontiguousarray(m.vertices, np.float32)
        ix = np.ascontiguousarray(m.indices, np.uint32)
        fm = np.ascontiguousarray(m.face_material, np.uint32)
        check(lib.rq_scene_create(_p(v), v.shape[0], _p(ix), m.n_tris, _p(fm),
                                  self.tri_kind, self.device, C.byref(self._h)))
        self._dirty = False

    def rebuild(self, bins: int = 0) -> None:
        """DynBVH::rebuild, done by the GPU binned-SAH builder."""
        if self._dirty or not self._h:
            self._upload()
        check(lib.rq_scene_build(self._h, bins))

    def update(self, rotate: bool = True) -> None:
        """DynBVH::update: the group's vertices moved (same triangles).
        rotate=True is the reference's update as it ships (refit, leaf
        re-splits and tree rotations, TREE_ROT 1); rotate=False refits the
        boxes and keeps the topology (TREE_ROT 0).  Both run on the GPU."""
        if self._dirty or not self._h:
            self.rebuild()
            return
        v = np.ascontiguousarray(self._group.vertices, np.float32)
        mode = RQ_UPDATE_ROTATE if rotate else RQ_UPDATE_REFIT
        check(lib.rq_scene_update_vertices_ex(self._h, _p(v), v.shape[0], mode))

    def update_device(self, vertices_ptr: int, rotate: bool = True, stream: int = 0) -> None:
        """update() with the new vertex positions already in device memory:
        a row-major array of 3 floats per vertex of the group (for a torch
        tensor, pass .contiguous().data_ptr())."""
        if self._dirty or not self._h:
            raise _lib.RQError(_lib.RQ_ERR_STATE, "no scene on the device to update")
        mode = RQ_UPDATE_ROTATE if rotate else RQ_UPDATE_REFIT
        check(lib.rq_scene_update_vertices_device(self._h, C.c_void_p(vertices_ptr),
                                                  self._group.vertices.shape[0], mode,
                                                  C.c_void_p(stream)))

    def update_state(self):
        """(costs, next_free): DynBVH::costs and DynBVH::nextFree, the state
        the next rotating update starts from."""
        nf = C.c_int()
        check(lib.rq_scene_update_state(self._h, None, 0, C.byref(nf)))
        costs = np.zeros(nf.value, np.float32)
        check(lib.rq_scene_update_state(self._h, _p(costs), costs.shape[0], C.byref(nf)))
        return costs, nf.value

    def importTree(self, tree) -> None:
        """Reference tree given field by field (oracle Tree or compatible)."""
        if self._dirty or not self._h:
            self._upload()
        b = np.ascontiguousarray(tree.bounds, np.float32)
        c = np.ascontiguousarray(tree.child, np.int32)
        ch = np.ascontiguousarray(tree.children, np.int32)
        ax = np.ascontiguousarray(tree.axis, np.uint8)
        lc = np.ascontiguousarray(tree.left_cheaper, np.uint8)
        ids = np.ascontiguousarray(tree.ids, np.int32)
        check(lib.rq_scene_import_tree(self._h, ch.shape[0], _p(b), _p(c), _p(ch), _p(ax),
                                       _p(lc), _p(ids)))

    def importBlob(self, blob: bytes) -> None:
        if self._dirty or not self._h:
            self._upload()
        buf = C.create_string_buffer(blob, len(blob))
        check(lib.rq_scene_import_dynbvh(self._h, buf, len(blob)))

    def buildFromFile(self, path: str) -> bool:
        """DynBVH::buildFromFile: the saveToFile byte stream."""
        try:
            with open(path, "rb") as f:
                blob = f.read()
        except OSError:
            return False
        self.importBlob(blob)
        return True

    def exportBlob(self) -> bytes:
        n = C.c_size_t()
        check(lib.rq_scene_export_dynbvh(self._h, None, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        check(lib.rq_scene_export_dynbvh(self._h, buf, C.byref(n)))
        return buf.raw[: n.value]

    def saveToFile(self, path: str) -> bool:
        with open(path, "wb") as f:
            f.write(self.exportBlob())
        return True

    def computeBounds(self):
        return self._group.bounds()

    def sahCost(self) -> float:
        c = C.c_double()
        check(lib.rq_scene_sah_cost(self._h, C.byref(c)))
        return c.value

    def info(self) -> SceneInfo:
        a, b, d = C.c_int(), C.c_int(), C.c_int()
        nb = C.c_size_t()
        check(lib.rq_scene_info(self._h, C.byref(a), C.byref(b), C.byref(d), C.byref(nb)))
        return SceneInfo(a.value, b.value, d.value, nb.value)

    def intersect(self, rays: RayBatch) -> None:
        """DynBVH::intersect over a host batch (copies in and out)."""
        n = len(rays)
        flags = RQ_ANYHIT if rays.getFlag(RQ_ANYHIT) else RQ_CLOSEST
        t = np.empty(n, np.float32)
        fn, h = lib.rq_trace, self._h
        if self._mode == self.Resident:
            if not self._ch:
                check(lib.rq_channel_create(self._h, 0, 0, C.byref(self._ch)))
            fn, h = lib.rq_channel_trace, self._ch
        check(fn(h, n, _p(rays.org), _p(rays.dir), _p(rays.minT), flags,
                 _p(t), _p(rays.hitPrim), _p(rays.u), _p(rays.v)))
        rays.minT[:] = t

    def intersect_device(self, n: int, org_ptr: int, dir_ptr: int, tmax_ptr: int,
                         anyhit: bool, t_ptr: int, prim_ptr: int, u_ptr: int = 0,
                         v_ptr: int = 0, stream: int = 0) -> None:
        """Query over device arrays already in HBM (raw pointers), enqueued on
        `stream` without synchronising."""
        check(lib.rq_trace_device(self._h, n, C.c_void_p(org_ptr), C.c_void_p(dir_ptr),
                                  C.c_void_p(tmax_ptr), RQ_ANYHIT if anyhit else RQ_CLOSEST,
                                  C.c_void_p(t_ptr), C.c_void_p(prim_ptr),
                                  C.c_void_p(u_ptr or None), C.c_void_p(v_ptr or None),
                                  C.c_void_p(stream or None)))

    def set_launch_config(self, anyhit: bool, block_threads=128, blocks_per_sm=0,
                          refill_threshold=8, persistent=True, stage=None,
                          reg_stack=0, node_layout=0) -> None:
        """Launch shape of ray queries (closest / any hit), or with
        stage=RQ_PATH_EXTEND / RQ_PATH_SHADE of a path-tracer stage
        (reg_stack: traversal-stack entries kept in registers, 0/1/2/4;
        node_layout: RQ_LAYOUT_* order of the records the path stages read)."""
        cfg = _lib.LaunchConfig(block_threads, blocks_per_sm, refill_threshold, int(persistent),
                                reg_stack, node_layout)
        flags = stage if stage is not None else (RQ_ANYHIT if anyhit else RQ_CLOSEST)
        check(lib.rq_set_launch_config(self._h, flags, C.byref(cfg)))

    def get_launch_config(self, anyhit: bool, stage=None) -> dict:
        cfg = _lib.LaunchConfig()
        flags = stage if stage is not None else (RQ_ANYHIT if anyhit else RQ_CLOSEST)
        check(lib.rq_get_launch_config(self._h, flags, C.byref(cfg)))
        return dict(block_threads=cfg.block_threads, blocks_per_sm=cfg.blocks_per_sm,
                    refill_threshold=cfg.refill_threshold, persistent=bool(cfg.persistent),
                    reg_stack=cfg.reg_stack, node_layout=cfg.node_layout)

    # -- frame path -----------------------------------------------------------
    @staticmethod
    def whitted_params(scene, materials=None) -> "_lib.WhittedParams":
        """rq_whitted_params for a scenes.WhittedScene (arrays kept alive on
        the returned object)."""
        p = _lib.WhittedParams()
        cam = scene.camera
        p.eye[:] = cam.eye
        p.lookat[:] = cam.lookat
        p.up[:] = cam.up
        p.hfov, p.vfov = cam.hfov, cam.vfov
        p.xres, p.yres = scene.xres, scene.yres
        lights = np.array([list(l.position) + list(l.color) for l in scene.lights],
                          np.float32).reshape(-1, 6)
        mats = np.ascontiguousarray(scene.mesh.materials if materials is None else materials,
                                    np.float32)
        p.n_lights = lights.shape[0]
        p.lights = lights.ctypes.data
        p.ambient[:] = scene.ambient
        p.background[:] = scene.background
        p.n_materials = mats.shape[0]
        p.material_rgb = mats.ctypes.data
        fill_environment(p.environment, getattr(scene, "environment", None))
        p._keep = (lights, mats)
        return p

    def render_whitted(self, scene):
        """Raytracer::traceEyeRays over a whole frame; host outputs."""
        p = self.whitted_params(scene)
        npx = scene.xres * scene.yres
        rgb = np.zeros((npx, 3), np.float32)
        t = np.zeros(npx, np.float32)
        prim = np.zeros(npx, np.int32)
        ns = C.c_uint64()
        check(lib.rq_render_whitted(self._h, C.byref(p), _p(rgb), _p(t), _p(prim), C.byref(ns)))
        return dict(rgb=rgb, t=t, prim=prim, shadow_rays=int(ns.value))

    def render_whitted_device(self, params, rgb_ptr: int, t_ptr: int, prim_ptr: int,
                              shadow_ptr: int = 0, stream: int = 0) -> None:
        check(lib.rq_render_whitted_device(self._h, C.byref(params), C.c_void_p(rgb_ptr),
                                           C.c_void_p(t_ptr), C.c_void_p(prim_ptr),
                                           C.c_void_p(shadow_ptr or None),
                                           C.c_void_p(stream or None)))

    @staticmethod
    def frame_params(scene, materials=None) -> "_lib.FrameParams":
        """rq_frame_params for a supersampled frame (any scene object with
        camera, lights, ambient, background, xres, yres, spp, seed, and
        optionally Phong `specular` / `specpow` per material)."""
        p = _lib.FrameParams()
        mats = getattr(scene, "materials", None) if materials is None else materials
        w = GpuDynBVH.whitted_params(scene, mats)
        p.whitted = w
        p.spp = int(scene.spp)
        p.seed = int(scene.seed)
        keep = list(w._keep)
        specpow = getattr(scene, "specpow", None)
        if specpow is not None:
            sp = np.ascontiguousarray(specpow, np.int32)
            ks = np.ascontiguousarray(scene.specular, np.float32)
            p.material_specular = ks.ctypes.data
            p.material_specpow = sp.ctypes.data
            keep += [sp, ks]
            refl = getattr(scene, "reflectivity", None)
            if refl is not None:
                rf = np.ascontiguousarray(refl, np.float32)
                p.material_reflectivity = rf.ctypes.data
                # RenderParameters defaults (Interface/RenderParameters.h)
                p.max_depth = int(getattr(scene, "max_depth", 15))
                p.importance_cutoff = float(getattr(scene, "importance_cutoff", 0.01))
                keep.append(rf)
        p._keep = keep
        return p

    def render_frame(self, scene, materials=None):
        """Supersampled Whitted frame (spp jittered samples per pixel,
        averaged) over this scene; host outputs."""
        p = self.frame_params(scene, materials)
        rgb = np.zeros((scene.xres * scene.yres, 3), np.float32)
        ns = C.c_uint64()
        check(lib.rq_render_frame(self._h, C.byref(p), _p(rgb), C.byref(ns)))
        return dict(rgb=rgb, shadow_rays=int(ns.value))

    def render_frame_device(self, params, rgb_ptr: int, shadow_ptr: int = 0,
                            stream: int = 0) -> None:
        check(lib.rq_render_frame_device(self._h, C.byref(params), C.c_void_p(rgb_ptr),
                                         C.c_void_p(shadow_ptr or None),
                                         C.c_void_p(stream or None)))

    def intersect_device_ex(self, n: int, org_ptr: int, dir_ptr: int, tmax_ptr: int,
                            anyhit: bool, t_ptr: int, prim_ptr: int, u_ptr: int = 0,
                            v_ptr: int = 0, inst_ptr: int = 0, stream: int = 0) -> None:
        """intersect_device plus the hit instance per ray (-1: none)."""
        check(lib.rq_trace_device_ex(self._h, n, C.c_void_p(org_ptr), C.c_void_p(dir_ptr),
                                     C.c_void_p(tmax_ptr), RQ_ANYHIT if anyhit else RQ_CLOSEST,
                                     C.c_void_p(t_ptr), C.c_void_p(prim_ptr),
                                     C.c_void_p(u_ptr or None), C.c_void_p(v_ptr or None),
                                     C.c_void_p(inst_ptr or None), C.c_void_p(stream or None)))

    def set_stage_events(self, events) -> None:
        """events: list of torch.cuda.Event (created with timing enabled and
        recorded at least once, which is when torch creates the CUDA event),
        or []."""
        if not events:
            check(lib.rq_set_stage_events(self._h, None, 0))
            return
        arr = (C.c_void_p * len(events))(*[e.cuda_event for e in events])
        self._events_keep = (arr, events)
        check(lib.rq_set_stage_events(self._h, arr, len(events)))

    @staticmethod
    def path_params(scene, chunk_paths: int = 0) -> "_lib.PathParams":
        """rq_path_params for a scenes.PathScene."""
        p = _lib.PathParams()
        cam = scene.camera
        p.eye[:] = cam.eye
        p.lookat[:] = cam.lookat
        p.up[:] = cam.up
        p.hfov, p.vfov = cam.hfov, cam.vfov
        p.xres, p.yres, p.spp = scene.xres, scene.yres, scene.spp
        p.max_depth, p.rr_depth, p.seed = scene.max_depth, scene.rr_depth, scene.seed
        L = scene.light
        p.light_anchor[:] = L.anchor
        p.light_v1[:] = L.v1
        p.light_v2[:] = L.v2
        p.light_color[:] = L.color
        p.background[:] = scene.background
        p.ambient[:] = getattr(scene, "ambient", (0.0, 0.0, 0.0))
        mats = np.ascontiguousarray(scene.mesh.materials, np.float32)
        p.n_materials = mats.shape[0]
        p.material_rgb = mats.ctypes.data
        p.chunk_paths = chunk_paths
        fill_environment(p.environment, getattr(scene, "environment", None))
        p._keep = (mats,)
        return p

    def render_path(self, scene, chunk_paths: int = 0):
        """KajiyaPathtracer frame; host outputs (rgb per pixel, ray counts)."""
        p = self.path_params(scene, chunk_paths)
        rgb = np.zeros((scene.xres * scene.yres, 3), np.float32)
        counts = (C.c_uint64 * 2)()
        check(lib.rq_render_path(self._h, C.byref(p), _p(rgb), counts))
        return dict(rgb=rgb, rays=int(counts[0]), shadow_rays=int(counts[1]))

    def render_path_device(self, params, rgb_ptr: int, counts_ptr: int = 0,
                           stream: int = 0) -> None:
        check(lib.rq_render_path_device(self._h, C.byref(params), C.c_void_p(rgb_ptr),
                                        C.c_void_p(counts_ptr or None),
                                        C.c_void_p(stream or None)))

    def set_path_debug(self, prim_ptr: int, org_ptr: int, dir_ptr: int, capacity: int) -> None:
        check(lib.rq_set_path_debug(self._h, C.c_void_p(prim_ptr or None),
                                    C.c_void_p(org_ptr or None), C.c_void_p(dir_ptr or None),
                                    capacity))

    def set_stats(self, counters_ptr: int) -> None:
        """Device uint64[4] receiving box/triangle test counts (0 = off)."""
        check(lib.rq_set_stats(self._h, C.c_void_p(counters_ptr or None)))

    def build_seconds(self) -> float:
        s = C.c_double()
        check(lib.rq_scene_build_seconds(self._h, C.byref(s)))
        return s.value

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def close(self) -> None:
        if self._ch:
            lib.rq_channel_destroy(self._ch)
            self._ch = C.c_void_p()
        if self._h:
            lib.rq_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class InstancedBVH(GpuDynBVH):
    """A top-level DynBVH over a Group of InstanceT objects
    (Model/Instances/InstanceT.cc) and nested DynBVHs: instance k places
    inner scene inst_scene[k] (a built GpuDynBVH) at translation[k], as an
    InstanceT (kind RQ_INST_TRANSLATE) or as the nested acceleration
    structure itself (RQ_INST_NESTED, zero translation).  The inner
    GpuDynBVHs must stay alive and keep their trees while this one is used.
    rebuild() builds the top-level tree on the GPU; importTree / importBlob
    take a reference top-level tree (object ids = instance indices)."""

    def __init__(self, inner: list, inst_scene, translation, kind=None):
        super().__init__(inner[0].tri_kind, inner[0].device)
        self._inner = list(inner)
        self._sc = np.ascontiguousarray(inst_scene, np.int32)
        self._tr = np.ascontiguousarray(translation, np.float32).reshape(-1, 3)
        self._kd = np.ascontiguousarray(
            np.zeros(self._sc.shape[0]) if kind is None else kind, np.int32)
        self._group = self._inner  # setGroup is not used: the instances are the group

    def setGroup(self, group) -> None:
        raise _lib.RQError(_lib.RQ_ERR_ARG, "an InstancedBVH takes its instances at construction")

    def _upload(self) -> None:
        self.close()
        hs = (C.c_void_p * len(self._inner))(*[b.handle.value for b in self._inner])
        self._hs = hs
        check(lib.rq_scene_create_instanced(hs, len(self._inner), _p(self._sc), _p(self._tr),
                                            _p(self._kd), self._sc.shape[0],
                                            C.byref(self._h)))
        self._dirty = False

    def rebuild(self, bins: int = 0) -> None:
        if not self._h:
            self._upload()  # builds the top-level tree
            if bins == 0:
                return
        check(lib.rq_scene_build(self._h, bins))

    @property
    def n_instances(self) -> int:
        return int(self._sc.shape[0])


def camera_basis(cam) -> np.ndarray:
    """PinholeCamera::setup basis (host-only C-ABI call)."""
    e = np.asarray(cam.eye, np.float32)
    la = np.asarray(cam.lookat, np.float32)
    up = np.asarray(cam.up, np.float32)
    out = np.zeros(12, np.float32)
    check(lib.rq_camera_basis(_p(e), _p(la), _p(up), cam.hfov, cam.vfov, _p(out)))
    return out


__all__ = ["GpuDynBVH", "InstancedBVH", "RayBatch", "RQ_TRI_WALD", "RQ_TRI_KS", "T_EPSILON", "MAXT"]
