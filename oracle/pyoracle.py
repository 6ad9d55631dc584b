"""Test infrastructure, not product code.

ctypes bindings for the two CPU checkers:
  * ``Restatement`` - oracle/rq_oracle.c, the per-ray C restatement of the
    reference's ray-query path (builds anywhere gcc exists);
  * ``Reference``   - oracle/_ref/libmanta_ref.so, the reference's own classes
    compiled from its sources by oracle/ref.mk, driven by
    oracle/ref_harness.cc.  Present only where that library was built.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmanta_ref.so")
REF_SSE_SO = os.path.join(HERE, "_ref", "libmanta_ref_sse.so")
DROPIN_SO = os.path.join(HERE, "_ref", "libmanta_dropin.so")
DROPIN_SSE_SO = os.path.join(HERE, "_ref", "libmanta_dropin_sse.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class _Env(C.Structure):
    """orq_env: ambient / background kinds, LinearBackground cdown and up."""
    _fields_ = [("ambient_kind", C.c_int), ("background_kind", C.c_int),
                ("down", C.c_float * 3), ("up", C.c_float * 3)]


def _env(scene):
    """orq_env for a scene's optional `environment` (None = constant forms)."""
    env = getattr(scene, "environment", None)
    if env is None:
        return None
    e = _Env()
    e.ambient_kind, e.background_kind = env.kinds()
    e.down[:] = env.background_down
    e.up[:] = env.background_up
    return C.byref(e)


@dataclass
class Tree:
    """Reference DynBVH node array, field by field (DynBVH.h:37-79)."""

    bounds: np.ndarray  # (N, 6) float32: min xyz, max xyz
    child: np.ndarray  # (N,) int32
    children: np.ndarray  # (N,) int32, leaf iff != 0
    axis: np.ndarray  # (N,) uint8
    left_cheaper: np.ndarray  # (N,) uint8
    ids: np.ndarray  # (T,) int32

    def arrays(self):
        return (np.ascontiguousarray(self.bounds, np.float32),
                np.ascontiguousarray(self.child, np.int32),
                np.ascontiguousarray(self.children, np.int32),
                np.ascontiguousarray(self.axis, np.uint8),
                np.ascontiguousarray(self.left_cheaper, np.uint8),
                np.ascontiguousarray(self.ids, np.int32))

    def save_npz(self, path):
        np.savez_compressed(path, bounds=self.bounds, child=self.child,
                            children=self.children, axis=self.axis,
                            left_cheaper=self.left_cheaper, ids=self.ids)

    @staticmethod
    def load_npz(path) -> "Tree":
        z = np.load(path)
        return Tree(z["bounds"], z["child"], z["children"], z["axis"],
                    z["left_cheaper"], z["ids"])


class DynTree:
    """A DynBVH as DynBVH::update sees it: the node array with room for
    `cap` nodes (the reference allocates 2 per object, DynBVH.cc:1680-1684),
    the per-node SAH costs, object_ids and nextFree."""

    def __init__(self, tree: Tree, n_objects: int, costs=None, next_free=None, cap=None):
        n = tree.children.shape[0]
        self.cap = int(cap if cap is not None else max(2 * n_objects, n))
        self.bounds = np.zeros((self.cap, 6), np.float32)
        self.child = np.zeros(self.cap, np.int32)
        self.children = np.zeros(self.cap, np.int32)
        self.axis = np.zeros(self.cap, np.uint8)
        self.left_cheaper = np.zeros(self.cap, np.uint8)
        self.costs = np.zeros(self.cap, np.float32)
        self.bounds[:n] = tree.bounds
        self.child[:n] = tree.child
        self.children[:n] = tree.children
        self.axis[:n] = tree.axis
        self.left_cheaper[:n] = tree.left_cheaper
        self.ids = np.ascontiguousarray(tree.ids, np.int32).copy()
        if costs is not None:
            self.costs[:len(costs)] = costs
        # nodes are allocated in pairs after the root
        self.next_free = int(next_free if next_free is not None else n)

    def tree(self, n=None) -> Tree:
        n = self.next_free if n is None else n
        return Tree(self.bounds[:n].copy(), self.child[:n].copy(), self.children[:n].copy(),
                    self.axis[:n].copy(), self.left_cheaper[:n].copy(), self.ids.copy())


class _OrqTree(C.Structure):
    _fields_ = [("bounds", C.c_void_p), ("child", C.c_void_p), ("children", C.c_void_p),
                ("axis", C.c_void_p), ("left_cheaper", C.c_void_p), ("ids", C.c_void_p),
                ("tri_kind", C.c_int), ("verts", C.c_void_p), ("idx", C.c_void_p),
                ("wald", C.c_void_p), ("face_mat", C.c_void_p)]


class _OrqWorld(C.Structure):
    _fields_ = [("top", C.c_void_p), ("inner", C.c_void_p), ("inst_scene", C.c_void_p),
                ("inst_T", C.c_void_p), ("inst_kind", C.c_void_p)]


class World:
    """A flat triangle scene or a two-level scene for the restatement: the
    top-level tree over instances of inner (tree, mesh) pairs.  Keeps every
    array it hands to C alive."""

    def __init__(self, rs: "Restatement", top_tree: Tree, top_mesh=None, inner=None,
                 inst_scene=None, translation=None, kind=None, tri_kind=0):
        self._keep = []
        self.inner_meshes = [m for _, m in inner] if inner else None
        if inner is None:
            self._top = self._tree(rs, top_tree, top_mesh, tri_kind)
            self.world = _OrqWorld(C.addressof(self._top), None, None, None, None)
        else:
            self._top = self._tree(rs, top_tree, None, tri_kind)
            arr = (_OrqTree * len(inner))()
            for i, (t, m) in enumerate(inner):
                arr[i] = self._tree(rs, t, m, tri_kind)
            self._inner = arr
            sc = np.ascontiguousarray(inst_scene, np.int32)
            tr = np.ascontiguousarray(translation, np.float32).reshape(-1, 3)
            kd = np.ascontiguousarray(kind if kind is not None else np.zeros(sc.shape[0]),
                                      np.int32)
            self._keep += [sc, tr, kd]
            self.world = _OrqWorld(C.addressof(self._top), C.addressof(arr), _ptr(sc).value,
                                   _ptr(tr).value, _ptr(kd).value)

    def _tree(self, rs, tree, mesh, tri_kind):
        b, c, ch, ax, lc, ids = tree.arrays()
        keep = [b, c, ch, ax, lc, ids]
        t = _OrqTree(_ptr(b).value, _ptr(c).value, _ptr(ch).value, _ptr(ax).value,
                     _ptr(lc).value, _ptr(ids).value, tri_kind, None, None, None, None)
        if mesh is not None:
            v = np.ascontiguousarray(mesh.vertices, np.float32)
            ix = np.ascontiguousarray(mesh.indices, np.uint32)
            fm = np.ascontiguousarray(mesh.face_material, np.uint32)
            w = rs.wald_setup(mesh) if tri_kind == 0 else None
            keep += [v, ix, fm, w]
            t.verts, t.idx, t.face_mat = _ptr(v).value, _ptr(ix).value, _ptr(fm).value
            t.wald = _ptr(w).value if w is not None else None
        self._keep += keep
        return t

    @property
    def ptr(self):
        return C.byref(self.world)


def build_restatement() -> str:
    if not os.path.exists(ORACLE_SO) or (
            os.path.getmtime(ORACLE_SO) < max(os.path.getmtime(os.path.join(HERE, f))
                                          for f in ("rq_oracle.c", "rq_oracle_update.c"))):
        subprocess.check_call(["make", "-s", "-f", os.path.join(HERE, "Makefile")],
                              cwd=os.path.dirname(HERE))
    return ORACLE_SO


class Restatement:
    """oracle/rq_oracle.c through ctypes."""

    def __init__(self):
        self.lib = C.CDLL(build_restatement())
        L = self.lib
        L.orq_wald_setup.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.orq_trace.argtypes = [C.c_void_p] * 10 + [C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 7
        L.orq_trace.argtypes = ([C.c_void_p] * 6 + [C.c_int] + [C.c_void_p] * 3 +
                                [C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 7)
        L.orq_top2.argtypes = ([C.c_void_p] * 6 + [C.c_int] + [C.c_void_p] * 3 +
                               [C.c_int] + [C.c_void_p] * 7)
        L.orq_sah_cost.argtypes = [C.c_void_p] * 3
        L.orq_sah_cost.restype = C.c_double
        L.orq_tree_costs.argtypes = [C.c_void_p] * 4
        L.orq_tree_costs.restype = C.c_float
        L.orq_tree_update.argtypes = ([C.c_void_p] * 7 + [C.c_int, C.c_void_p, C.c_void_p,
                                                          C.c_void_p, C.c_int, C.c_int])
        L.orq_camera_basis.argtypes = [C.c_void_p] * 3 + [C.c_float, C.c_float, C.c_void_p]
        L.orq_primary_rays.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.orq_render_whitted.argtypes = ([C.c_void_p] * 6 + [C.c_int] + [C.c_void_p] * 6 +
                                         [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 6)
        L.orq_render_whitted.restype = C.c_longlong
        L.orq_sincos_2pi.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.orq_render_path.argtypes = ([C.c_void_p] * 6 + [C.c_int] + [C.c_void_p] * 7 +
                                      [C.c_uint64, C.c_longlong, C.c_longlong] +
                                      [C.c_void_p] * 4)
        L.orq_trace_world.argtypes = ([C.c_void_p, C.c_int] + [C.c_void_p] * 3 + [C.c_int] +
                                      [C.c_void_p] * 6)
        L.orq_sample_coords.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_longlong,
                                        C.c_longlong, C.c_void_p, C.c_void_p]
        L.orq_render_frame.argtypes = ([C.c_void_p] * 5 + [C.c_int, C.c_float, C.c_void_p] +
                                       [C.c_int] * 3 + [C.c_uint64] +
                                       [C.c_void_p, C.c_int] + [C.c_void_p] * 2 +
                                       [C.c_int, C.c_int] + [C.c_void_p] * 5)
        L.orq_render_frame.restype = C.c_longlong

    def world(self, top_tree, top_mesh=None, inner=None, inst_scene=None, translation=None,
              kind=None, tri_kind=0) -> World:
        return World(self, top_tree, top_mesh, inner, inst_scene, translation, kind, tri_kind)

    def trace_world(self, world: World, org, dir, tmax, anyhit=False):
        n = int(tmax.shape[0])
        org = np.ascontiguousarray(org, np.float32)
        dir = np.ascontiguousarray(dir, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        hit = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        inst = np.zeros(n, np.int32)
        self.lib.orq_trace_world(world.ptr, n, _ptr(org), _ptr(dir), _ptr(tmax), int(anyhit),
                                 _ptr(hit), _ptr(t), _ptr(prim), _ptr(u), _ptr(v), _ptr(inst))
        return dict(hit=hit, t=t, prim=prim, u=u, v=v, inst=inst)

    def sample_coords(self, xres, yres, spp, seed, items=None):
        i0, i1 = items if items else (0, xres * yres * spp)
        px = np.zeros(i1 - i0, np.float32)
        py = np.zeros(i1 - i0, np.float32)
        self.lib.orq_sample_coords(xres, yres, spp, int(seed), i0, i1, _ptr(px), _ptr(py))
        return px, py

    def render_frame(self, world: World, scene, materials, rows=None, per_sample=False,
                     specular=None, specpow=None, reflectivity=None, max_depth=15,
                     cutoff=0.01):
        """Supersampled Whitted frame (any scene with camera, lights,
        ambient, background, xres, yres, spp, seed) over a world; materials
        with specpow >= 0 are Phong with the given specular colour and
        reflectivity (RenderParameters maxDepth / importanceCutoff)."""
        basis = self.camera_basis(scene.camera)
        xres, yres, spp = scene.xres, scene.yres, scene.spp
        y0, y1 = rows if rows else (0, yres)
        lights = np.array([list(l.position) + list(l.color) for l in scene.lights],
                          np.float32).reshape(-1, 6)
        amb = np.asarray(scene.ambient, np.float32)
        bg = np.asarray(scene.background, np.float32)
        mats = np.ascontiguousarray(materials, np.float32)
        spec = None if specpow is None else np.ascontiguousarray(specular, np.float32)
        spow = None if specpow is None else np.ascontiguousarray(specpow, np.int32)
        npx = (y1 - y0) * xres
        rgb = np.zeros((npx, 3), np.float32)
        srgb = np.zeros((npx * spp, 3), np.float32) if per_sample else None
        st = np.zeros(npx * spp, np.float32) if per_sample else None
        sp = np.zeros(npx * spp, np.int32) if per_sample else None
        refl = None if reflectivity is None else np.ascontiguousarray(reflectivity, np.float32)
        ns = self.lib.orq_render_frame(world.ptr, _ptr(mats), _ptr(spec), _ptr(spow), _ptr(refl),
                                       int(max_depth), float(cutoff), _ptr(basis), xres, yres, spp,
                                       int(scene.seed), _ptr(lights), lights.shape[0],
                                       _ptr(amb), _ptr(bg), y0, y1, _ptr(rgb), _ptr(srgb),
                                       _ptr(st), _ptr(sp), _env(scene))
        out = dict(rgb=rgb, shadow_rays=int(ns))
        if per_sample:
            out.update(sample_rgb=srgb, sample_t=st, sample_prim=sp)
        return out

    def sincos_2pi(self, u):
        u = np.ascontiguousarray(u, np.float32)
        c = np.zeros_like(u)
        s = np.zeros_like(u)
        self.lib.orq_sincos_2pi(_ptr(u), u.shape[0], _ptr(c), _ptr(s))
        return c, s

    def render_path(self, tree, scene, tri_kind=0, paths=None, debug=False):
        """Path-traced frame (restatement of the device wavefront).  Returns
        per-path radiance for paths [p0, p1), the pixel image when all paths
        are traced, ray counts and optionally per-bounce hit ids."""
        mesh = scene.mesh
        keep, args = self._scene_args(tree, mesh, tri_kind, None)
        basis = self.camera_basis(scene.camera)
        L = scene.light
        fp = np.concatenate([basis, np.asarray(L.anchor, np.float32),
                             np.asarray(L.v1, np.float32), np.asarray(L.v2, np.float32),
                             np.asarray(L.color, np.float32),
                             np.asarray(scene.background, np.float32),
                             np.asarray(getattr(scene, "ambient", (0.0, 0.0, 0.0)),
                                        np.float32)]).astype(np.float32)
        ip = np.array([scene.xres, scene.yres, scene.spp, scene.max_depth, scene.rr_depth],
                      np.int32)
        total = scene.xres * scene.yres * scene.spp
        p0, p1 = paths if paths else (0, total)
        rad = np.zeros((p1 - p0, 3), np.float32)
        counts = np.zeros(2, np.int64)
        dbg = np.full((scene.max_depth, total), -2, np.int32) if debug else None
        fm = np.ascontiguousarray(mesh.face_material, np.uint32)
        mats = np.ascontiguousarray(mesh.materials, np.float32)
        self.lib.orq_render_path(*args, _ptr(fm), _ptr(mats), _ptr(fp), _ptr(ip),
                                 int(scene.seed), p0, p1, _ptr(rad), _ptr(counts), _ptr(dbg),
                                 _env(scene))
        out = dict(rad=rad, rays=int(counts[0]), shadow_rays=int(counts[1]), prim=dbg)
        if paths is None:
            r = rad.reshape(-1, scene.spp, 3)
            acc = np.zeros((r.shape[0], 3), np.float32)
            for s_ in range(scene.spp):
                acc = (acc + r[:, s_]).astype(np.float32)
            out["rgb"] = (acc * np.float32(np.float32(1.0) / np.float32(scene.spp))).astype(np.float32)
        return out

    def wald_setup(self, mesh) -> np.ndarray:
        v = np.ascontiguousarray(mesh.vertices, np.float32)
        i = np.ascontiguousarray(mesh.indices, np.uint32)
        out = np.zeros((mesh.n_tris, 12), np.float32)
        self.lib.orq_wald_setup(_ptr(v), _ptr(i), mesh.n_tris, _ptr(out))
        return out

    def _scene_args(self, tree: Tree, mesh, tri_kind, wald):
        b, c, ch, ax, lc, ids = tree.arrays()
        v = np.ascontiguousarray(mesh.vertices, np.float32)
        ix = np.ascontiguousarray(mesh.indices, np.uint32)
        if wald is None and tri_kind == 0:
            wald = self.wald_setup(mesh)
        keep = (b, c, ch, ax, lc, ids, v, ix, wald)
        args = [_ptr(b), _ptr(c), _ptr(ch), _ptr(ax), _ptr(lc), _ptr(ids), tri_kind,
                _ptr(v), _ptr(ix), _ptr(wald) if wald is not None else None]
        return keep, args

    def trace(self, tree, mesh, org, dir, tmax, anyhit=False, tri_kind=0,
              wald=None, counts=False):
        n = int(tmax.shape[0])
        org = np.ascontiguousarray(org, np.float32)
        dir = np.ascontiguousarray(dir, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        keep, args = self._scene_args(tree, mesh, tri_kind, wald)
        hit = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        nt = np.zeros(n, np.int32) if counts else None
        tt = np.zeros(n, np.int32) if counts else None
        self.lib.orq_trace(*args, n, _ptr(org), _ptr(dir), _ptr(tmax), int(anyhit),
                           _ptr(hit), _ptr(t), _ptr(prim), _ptr(u), _ptr(v),
                           _ptr(nt), _ptr(tt))
        out = dict(hit=hit, t=t, prim=prim, u=u, v=v)
        if counts:
            out["node_tests"] = nt
            out["tri_tests"] = tt
        return out

    def top2(self, tree, mesh, org, dir, tmax, tri_kind=0, wald=None):
        n = int(tmax.shape[0])
        org = np.ascontiguousarray(org, np.float32)
        dir = np.ascontiguousarray(dir, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        keep, args = self._scene_args(tree, mesh, tri_kind, wald)
        t1 = np.zeros(n, np.float32)
        t2 = np.zeros(n, np.float32)
        p1 = np.zeros(n, np.int32)
        p2 = np.zeros(n, np.int32)
        self.lib.orq_top2(*args, n, _ptr(org), _ptr(dir), _ptr(tmax),
                          _ptr(t1), _ptr(t2), _ptr(p1), _ptr(p2))
        return t1, t2, p1, p2

    def sah_cost(self, tree: Tree) -> float:
        b, c, ch, *_ = tree.arrays()
        return float(self.lib.orq_sah_cost(_ptr(b), _ptr(c), _ptr(ch)))

    def tree_costs(self, t: DynTree) -> float:
        """DynBVH::computeCost<true>(0) into t.costs (a rebuild's state)."""
        return float(self.lib.orq_tree_costs(_ptr(t.bounds), _ptr(t.child), _ptr(t.children),
                                             _ptr(t.costs)))

    def tree_update(self, t: DynTree, vertices, indices, rotate=True) -> None:
        """DynBVH::update(0, 1) of t in place after the vertices moved."""
        v = np.ascontiguousarray(vertices, np.float32)
        ix = np.ascontiguousarray(indices, np.uint32)
        nf = C.c_int(t.next_free)
        rc = self.lib.orq_tree_update(_ptr(t.bounds), _ptr(t.child), _ptr(t.children),
                                      _ptr(t.axis), _ptr(t.left_cheaper), _ptr(t.costs),
                                      _ptr(t.ids), t.cap, C.byref(nf), _ptr(v), _ptr(ix),
                                      ix.shape[0], int(rotate))
        if rc != 0:
            raise RuntimeError(f"orq_tree_update failed ({rc})")
        t.next_free = nf.value

    def camera_basis(self, cam) -> np.ndarray:
        e = np.asarray(cam.eye, np.float32)
        la = np.asarray(cam.lookat, np.float32)
        up = np.asarray(cam.up, np.float32)
        out = np.zeros(12, np.float32)
        self.lib.orq_camera_basis(_ptr(e), _ptr(la), _ptr(up), cam.hfov, cam.vfov, _ptr(out))
        return out

    def primary_rays(self, basis, xres, yres):
        n = xres * yres
        org = np.zeros((3, n), np.float32)
        dir = np.zeros((3, n), np.float32)
        b = np.ascontiguousarray(basis, np.float32)
        self.lib.orq_primary_rays(_ptr(b), xres, yres, _ptr(org), _ptr(dir))
        return org, dir

    def render_whitted(self, tree, scene, tri_kind=0, wald=None, rows=None):
        mesh = scene.mesh
        keep, args = self._scene_args(tree, mesh, tri_kind, wald)
        basis = self.camera_basis(scene.camera)
        xres, yres = scene.xres, scene.yres
        y0, y1 = rows if rows else (0, yres)
        lights = np.array([list(l.position) + list(l.color) for l in scene.lights], np.float32)
        amb = np.asarray(scene.ambient, np.float32)
        bg = np.asarray(scene.background, np.float32)
        fm = np.ascontiguousarray(mesh.face_material, np.uint32)
        mats = np.ascontiguousarray(mesh.materials, np.float32)
        npx = xres * yres
        rgb = np.zeros((npx, 3), np.float32)
        tp = np.zeros(npx, np.float32)
        pr = np.full(npx, -1, np.int32)
        lit = np.zeros(npx, np.int32)
        counts = np.zeros(4, np.int64)
        ns = self.lib.orq_render_whitted(*args, _ptr(fm), _ptr(mats), _ptr(basis), xres, yres,
                                         _ptr(lights), len(scene.lights), _ptr(amb), _ptr(bg),
                                         y0, y1, _ptr(rgb), _ptr(tp), _ptr(pr), _ptr(lit),
                                         _ptr(counts), _env(scene))
        return dict(rgb=rgb, t=tp, prim=pr, lit=lit, shadow_rays=int(ns),
                    primary_node_tests=int(counts[0]), primary_tri_tests=int(counts[1]),
                    shadow_node_tests=int(counts[2]), shadow_tri_tests=int(counts[3]))


class Reference:
    """The reference's own classes (oracle/_ref), through ref_harness.cc."""

    def __init__(self, sse: bool = False, path: str | None = None):
        path = path or (REF_SSE_SO if sse else REF_SO)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        # keep the process exit status (the reference's thread library would
        # replace it with 0 at exit)
        L.mref_keep_exit_status()
        L.mref_scene_create.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.mref_scene_create.restype = C.c_void_p
        L.mref_scene_destroy.argtypes = [C.c_void_p]
        L.mref_tree_count.argtypes = [C.c_void_p] * 4
        L.mref_tree_export.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 6
        L.mref_tree_save.argtypes = [C.c_void_p, C.c_char_p]
        L.mref_tree_state.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.mref_read_obj.argtypes = [C.c_char_p, C.c_int] + [C.c_void_p] * 8 + [C.c_int] * 3
        L.mref_tree_cost.argtypes = [C.c_void_p]
        L.mref_tree_cost.restype = C.c_double
        L.mref_intersect.argtypes = ([C.c_void_p, C.c_int] + [C.c_void_p] * 3 +
                                     [C.c_int, C.c_int] + [C.c_void_p] * 5)
        L.mref_camera_basis.argtypes = [C.c_void_p] * 3 + [C.c_float, C.c_float, C.c_void_p]
        L.mref_render.argtypes = ([C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 2 + [C.c_int] +
                                  [C.c_void_p] * 2 + [C.c_int] + [C.c_void_p] * 5)
        L.mref_node_size.restype = C.c_int
        L.mref_intersect_mt.argtypes = ([C.c_void_p, C.c_int] + [C.c_void_p] * 3 +
                                        [C.c_int, C.c_int] + [C.c_void_p] * 4)
        if hasattr(L, "mref_scene_use_gpu"):
            L.mref_scene_use_gpu.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_char_p]
            L.mref_scene_gpu_options.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.mref_scene_gpu_as_primitive.argtypes = [C.c_void_p]
        L.mref_render_path.argtypes = ([C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                        C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_uint,
                                        C.c_void_p, C.c_void_p, C.c_void_p])
        L.mref_intersect2.argtypes = ([C.c_void_p, C.c_int] + [C.c_void_p] * 3 +
                                      [C.c_int, C.c_int] + [C.c_void_p] * 6)
        L.mref_scene_create_instanced.argtypes = ([C.c_void_p, C.c_int] + [C.c_void_p] * 3 +
                                                  [C.c_int])
        L.mref_scene_create_instanced.restype = C.c_void_p
        L.mref_scene_set_phong.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float]
        L.mref_scene_set_render_parameters.argtypes = [C.c_void_p, C.c_int, C.c_float]
        L.mref_scene_set_environment.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                                 C.c_void_p]
        L.mref_read_ply.argtypes = ([C.c_char_p, C.c_void_p, C.c_int] + [C.c_void_p] * 5 +
                                    [C.c_int, C.c_int])
        L.mref_scene_update_vertices.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.mref_render_coords.argtypes = ([C.c_void_p, C.c_int] + [C.c_void_p] * 4 + [C.c_int] +
                                         [C.c_void_p] * 2 + [C.c_int] + [C.c_void_p] * 4)

    @staticmethod
    def available(sse: bool = False) -> bool:
        return os.path.exists(REF_SSE_SO if sse else REF_SO)

    def scene(self, mesh, tri_kind=0) -> "RefScene":
        return RefScene(self, mesh, tri_kind)

    def instanced(self, inner: list, inst_scene, translation, kind=None) -> "RefScene":
        """Top-level DynBVH over InstanceT (kind 0) / nested DynBVH (kind 1)
        objects of the inner RefScenes."""
        return RefScene(self, None, 0, inner=(inner, inst_scene, translation, kind))

    def read_obj(self, path, tri_kind=0):
        """Manta::ObjGroup over glm: (vertices, indices, face_material,
        material kinds, material values [n, 13]: Kd rgb, Ks rgb, Ns, Ni, d,
        filter rgb, reflectivity), or None when the reader fails."""
        nv, nt, nm = C.c_int(), C.c_int(), C.c_int()
        L = self.lib
        rc = L.mref_read_obj(str(path).encode(), tri_kind, C.byref(nv), C.byref(nt), C.byref(nm),
                             None, None, None, None, None, 0, 0, 0)
        if rc != 0:
            return None
        v = np.zeros((nv.value, 3), np.float32)
        ix = np.zeros((nt.value, 3), np.uint32)
        fm = np.zeros(nt.value, np.uint32)
        kind = np.zeros(nm.value, np.int32)
        vals = np.zeros((nm.value, 13), np.float32)
        rc = L.mref_read_obj(str(path).encode(), tri_kind, C.byref(nv), C.byref(nt), C.byref(nm),
                             _ptr(v), _ptr(ix), _ptr(fm), _ptr(kind), _ptr(vals), v.shape[0],
                             ix.shape[0], kind.shape[0])
        if rc != 0:
            return None
        return v, ix, fm, kind, vals

    def read_ply(self, path, transform=None, tri_kind=0):
        """Manta::readPlyFile into a fresh Mesh: (vertices, indices,
        face_material), or None when the reader fails."""
        t = None if transform is None else np.ascontiguousarray(transform, np.float32).reshape(12)
        nv, nt = C.c_int(), C.c_int()
        rc = self.lib.mref_read_ply(str(path).encode(), _ptr(t), tri_kind, C.byref(nv),
                                    C.byref(nt), None, None, None, 0, 0)
        if rc != 0:
            return None
        v = np.zeros((nv.value, 3), np.float32)
        ix = np.zeros((nt.value, 3), np.uint32)
        fm = np.zeros(nt.value, np.uint32)
        rc = self.lib.mref_read_ply(str(path).encode(), _ptr(t), tri_kind, C.byref(nv),
                                    C.byref(nt), _ptr(v), _ptr(ix), _ptr(fm), v.shape[0],
                                    ix.shape[0])
        if rc != 0:
            return None
        return v, ix, fm

    def camera_basis(self, cam) -> np.ndarray:
        e = np.asarray(cam.eye, np.float32)
        la = np.asarray(cam.lookat, np.float32)
        up = np.asarray(cam.up, np.float32)
        out = np.zeros(12, np.float32)
        self.lib.mref_camera_basis(_ptr(e), _ptr(la), _ptr(up), cam.hfov, cam.vfov, _ptr(out))
        return out


class RefScene:
    def __init__(self, ref: Reference, mesh, tri_kind=0, inner=None):
        self.ref = ref
        self.mesh = mesh
        if inner is not None:
            scenes, inst_scene, translation, kind = inner
            hs = (C.c_void_p * len(scenes))(*[x.h for x in scenes])
            sc = np.ascontiguousarray(inst_scene, np.int32)
            tr = np.ascontiguousarray(translation, np.float32).reshape(-1, 3)
            kd = np.ascontiguousarray(kind if kind is not None else np.zeros(sc.shape[0]),
                                      np.int32)
            self._keep = (scenes, hs, sc, tr, kd)
            self.h = ref.lib.mref_scene_create_instanced(hs, len(scenes), _ptr(sc), _ptr(tr),
                                                         _ptr(kd), sc.shape[0])
            if not self.h:
                raise RuntimeError("reference instanced scene build failed")
            return
        v = np.ascontiguousarray(mesh.vertices, np.float32)
        ix = np.ascontiguousarray(mesh.indices, np.uint32)
        fm = np.ascontiguousarray(mesh.face_material, np.uint32)
        mats = np.ascontiguousarray(mesh.materials, np.float32)
        self._keep = (v, ix, fm, mats)
        self.h = ref.lib.mref_scene_create(_ptr(v), v.shape[0], _ptr(ix), mesh.n_tris,
                                           _ptr(fm), _ptr(mats), mats.shape[0], tri_kind)
        if not self.h:
            raise RuntimeError("reference scene build failed")

    def set_phong(self, material: int, specular, specpow: int, reflectivity: float = 0.0) -> None:
        """Material `material` becomes a Phong with its diffuse colour and
        the given specular colour, exponent and reflectivity (0: none)."""
        sp = np.ascontiguousarray(specular, np.float32)
        if self.ref.lib.mref_scene_set_phong(self.h, material, _ptr(sp), int(specpow),
                                             float(reflectivity)) != 0:
            raise RuntimeError("mref_scene_set_phong failed")

    def set_render_parameters(self, max_depth: int, cutoff: float) -> None:
        """RenderParameters maxDepth / importanceCutoff of later renders."""
        self.ref.lib.mref_scene_set_render_parameters(self.h, int(max_depth), float(cutoff))

    def set_environment(self, env) -> None:
        """EyeAmbient / LinearBackground for later renders (a
        scenes.Environment; None = ConstantAmbient / ConstantBackground)."""
        if env is None:
            self.ref.lib.mref_scene_set_environment(self.h, 0, 0, None, None)
            return
        a, b = env.kinds()
        down = np.asarray(env.background_down, np.float32)
        up = np.asarray(env.background_up, np.float32)
        self.ref.lib.mref_scene_set_environment(self.h, a, b, _ptr(down), _ptr(up))

    def update_vertices(self, vertices) -> None:
        """Animated mesh: new vertex positions, WaldTriangle::update and
        DynBVH::update (the reference's refit)."""
        v = np.ascontiguousarray(vertices, np.float32)
        if self.ref.lib.mref_scene_update_vertices(self.h, _ptr(v), v.shape[0]) != 0:
            raise RuntimeError("mref_scene_update_vertices failed")

    def use_gpu(self, device=0, tri_kind=0, tree_file=None):
        """Drop-in library only: trace with rfmanta_b200's GpuDynBVH."""
        rc = self.ref.lib.mref_scene_use_gpu(self.h, device, tri_kind,
                                             tree_file.encode() if tree_file else None)
        if rc != 0:
            raise RuntimeError(f"mref_scene_use_gpu failed ({rc})")

    def gpu_as_primitive(self):
        """Drop-in library only: trace through a reference Group holding a
        GpuMeshPrimitive (the Primitive surface) instead of the bare
        GpuDynBVH."""
        if self.ref.lib.mref_scene_gpu_as_primitive(self.h) != 0:
            raise RuntimeError("mref_scene_gpu_as_primitive: the scene is not on the drop-in")

    def gpu_options(self, batching=True, gpu_shadows=False, mode=None):
        """Drop-in library only: packets through the submission queue
        (batching) or one round trip each, or `mode` 0 / 1 / 2 = per call /
        queue / resident packet channel; GpuHardShadows instead of
        HardShadows."""
        m = int(batching) if mode is None else int(mode)
        if self.ref.lib.mref_scene_gpu_options(self.h, m, int(gpu_shadows)) != 0:
            raise RuntimeError("mref_scene_gpu_options: the scene is not on the drop-in")

    def close(self):
        if self.h:
            self.ref.lib.mref_scene_destroy(self.h)
            self.h = None

    def tree(self) -> Tree:
        used, alloc, nids = C.c_int(), C.c_int(), C.c_int()
        self.ref.lib.mref_tree_count(self.h, C.byref(used), C.byref(alloc), C.byref(nids))
        n = used.value
        b = np.zeros((n, 6), np.float32)
        c = np.zeros(n, np.int32)
        ch = np.zeros(n, np.int32)
        ax = np.zeros(n, np.uint8)
        lc = np.zeros(n, np.uint8)
        ids = np.zeros(nids.value, np.int32)
        self.ref.lib.mref_tree_export(self.h, n, _ptr(b), _ptr(c), _ptr(ch), _ptr(ax),
                                      _ptr(lc), _ptr(ids))
        return Tree(b, c, ch, ax, lc, ids)

    def dyn_tree(self) -> DynTree:
        """The tree with its costs and nextFree (no call may run
        computeCost in between: it rewrites the costs)."""
        used, alloc, nids = C.c_int(), C.c_int(), C.c_int()
        self.ref.lib.mref_tree_count(self.h, C.byref(used), C.byref(alloc), C.byref(nids))
        costs = np.zeros(used.value, np.float32)
        nf = C.c_int()
        if self.ref.lib.mref_tree_state(self.h, _ptr(costs), used.value, C.byref(nf)) != 0:
            raise RuntimeError("mref_tree_state failed")
        return DynTree(self.tree(), nids.value, costs=costs, next_free=nf.value,
                       cap=alloc.value)

    def save_blob(self, path: str):
        if self.ref.lib.mref_tree_save(self.h, path.encode()) != 0:
            raise RuntimeError("saveToFile failed")

    def sah_cost(self) -> float:
        return float(self.ref.lib.mref_tree_cost(self.h))

    def intersect(self, org, dir, tmax, anyhit=False, packet=64):
        n = int(tmax.shape[0])
        org = np.ascontiguousarray(org, np.float32)
        dir = np.ascontiguousarray(dir, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        hit = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        self.ref.lib.mref_intersect(self.h, n, _ptr(org), _ptr(dir), _ptr(tmax), int(anyhit),
                                    packet, _ptr(hit), _ptr(t), _ptr(prim), _ptr(u), _ptr(v))
        return dict(hit=hit, t=t, prim=prim, u=u, v=v)

    def intersect2(self, org, dir, tmax, anyhit=False, packet=64):
        """intersect plus the hit instance (-1: none or not an InstanceT);
        u/v are 0 for InstanceT hits (the reference keeps them in the
        instance's own packet)."""
        n = int(tmax.shape[0])
        org = np.ascontiguousarray(org, np.float32)
        dir = np.ascontiguousarray(dir, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        out = {k: np.zeros(n, np.int32 if k in ("hit", "prim", "inst") else np.float32)
               for k in ("hit", "t", "prim", "u", "v", "inst")}
        self.ref.lib.mref_intersect2(self.h, n, _ptr(org), _ptr(dir), _ptr(tmax), int(anyhit),
                                     packet, *[_ptr(out[k]) for k in
                                               ("hit", "t", "prim", "u", "v", "inst")])
        return out

    def render_coords(self, scene, px, py, nthreads=1):
        """Raytracer::traceEyeRays at the given image coordinates (one eye
        ray each); per-ray colour, primary t and triangle id."""
        cam = scene.camera
        args = np.array(list(cam.eye) + list(cam.lookat) + list(cam.up) +
                        [cam.hfov, cam.vfov, 0.0], np.float32)
        lights = np.array([list(l.position) + list(l.color) for l in scene.lights],
                          np.float32).reshape(-1, 6)
        amb = np.asarray(scene.ambient, np.float32)
        bg = np.asarray(scene.background, np.float32)
        px = np.ascontiguousarray(px, np.float32)
        py = np.ascontiguousarray(py, np.float32)
        n = px.shape[0]
        rgb = np.zeros((n, 3), np.float32)
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32)
        nsr = C.c_longlong()
        self.ref.lib.mref_render_coords(self.h, n, _ptr(px), _ptr(py), _ptr(args), _ptr(lights),
                                        lights.shape[0], _ptr(amb), _ptr(bg), nthreads,
                                        _ptr(rgb), _ptr(t), _ptr(prim), C.byref(nsr))
        return dict(rgb=rgb, t=t, prim=prim, shadow_rays=nsr.value)

    def intersect_mt(self, org, dir, tmax, anyhit=False, nthreads=1):
        """DynBVH::intersect on 64-ray packets over N threads; returns the
        outputs and the wall seconds."""
        n = int(tmax.shape[0])
        org = np.ascontiguousarray(org, np.float32)
        dir = np.ascontiguousarray(dir, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        hit = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.int32)
        secs = C.c_double()
        self.ref.lib.mref_intersect_mt(self.h, n, _ptr(org), _ptr(dir), _ptr(tmax), int(anyhit),
                                       nthreads, _ptr(hit), _ptr(t), _ptr(prim), C.byref(secs))
        return dict(hit=hit, t=t, prim=prim, seconds=secs.value)

    def render(self, scene, nthreads=1, want_ids=True):
        cam = scene.camera
        args = np.array(list(cam.eye) + list(cam.lookat) + list(cam.up) +
                        [cam.hfov, cam.vfov, 0.0], np.float32)
        lights = np.array([list(l.position) + list(l.color) for l in scene.lights], np.float32)
        amb = np.asarray(scene.ambient, np.float32)
        bg = np.asarray(scene.background, np.float32)
        npx = scene.xres * scene.yres
        rgb = np.zeros((npx, 3), np.float32)
        tp = np.zeros(npx, np.float32) if want_ids else None
        pr = np.zeros(npx, np.int32) if want_ids else None
        secs = C.c_double()
        nsr = C.c_longlong()
        self.ref.lib.mref_render(self.h, scene.xres, scene.yres, _ptr(args), _ptr(lights),
                                 len(scene.lights), _ptr(amb), _ptr(bg), nthreads, _ptr(rgb),
                                 _ptr(tp), _ptr(pr), C.byref(secs), C.byref(nsr))
        return dict(rgb=rgb, t=tp, prim=pr, seconds=secs.value, shadow_rays=nsr.value)

    def render_path(self, scene, nthreads=1):
        """KajiyaPathtracer frame (reference defaults) over this scene."""
        cam = scene.camera
        args = np.array(list(cam.eye) + list(cam.lookat) + list(cam.up) +
                        [cam.hfov, cam.vfov], np.float32)
        L = scene.light
        light = np.array(list(L.anchor) + list(L.v1) + list(L.v2) + list(L.color), np.float32)
        bg = np.asarray(list(scene.background) +
                        list(getattr(scene, "ambient", (0.0, 0.0, 0.0))), np.float32)
        rgb = np.zeros((scene.xres * scene.yres, 3), np.float32)
        secs = C.c_double()
        rays = C.c_longlong()
        self.ref.lib.mref_render_path(self.h, scene.xres, scene.yres, _ptr(args), scene.spp,
                                      scene.max_depth, _ptr(light), _ptr(bg), nthreads,
                                      int(scene.seed), _ptr(rgb), C.byref(secs), C.byref(rays))
        return dict(rgb=rgb, seconds=secs.value, rays=rays.value)
