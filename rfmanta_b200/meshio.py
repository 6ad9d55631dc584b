"""Mesh files through the C ABI into a scenes.Mesh ready for
GpuDynBVH.setGroup: PLY (rq_mesh_read_ply, the reader of Manta::readPlyFile,
Model/Readers/PlyReader.cc) and Wavefront OBJ + MTL (rq_mesh_read_obj, the
reader of Manta::ObjGroup, Model/Groups/ObjGroup.cc)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib
from .scenes import Mesh


def read_ply(path: str, transform=None, material: int = 0,
             materials: np.ndarray | None = None) -> Mesh:
    """Reads a PLY file; `transform` is a 3x4 matrix (None = identity)
    applied to every vertex, `material` the face material of every triangle
    and `materials` the mesh's material table (default: one white
    Lambertian, as the reference's reader adds)."""
    h = C.c_void_p()
    t = None if transform is None else np.ascontiguousarray(transform, np.float32).reshape(12)
    check(lib.rq_mesh_read_ply(str(path).encode(), None if t is None else t.ctypes.data,
                               int(material), C.byref(h)))
    try:
        nv, nt = C.c_int(), C.c_int()
        check(lib.rq_mesh_info(h, C.byref(nv), C.byref(nt)))
        v = np.zeros((nv.value, 3), np.float32)
        ix = np.zeros((nt.value, 3), np.uint32)
        fm = np.zeros(nt.value, np.uint32)
        check(lib.rq_mesh_copy(h, v.ctypes.data, ix.ctypes.data, fm.ctypes.data))
    finally:
        lib.rq_mesh_destroy(h)
    mats = (np.ones((int(material) + 1, 3), np.float32) if materials is None
            else np.ascontiguousarray(materials, np.float32).reshape(-1, 3))
    return Mesh(v, ix, fm, mats)


class ObjMaterials:
    """ObjGroup's material table: per entry the kind (_lib.RQ_MAT_*),
    diffuse and specular rgb, Phong exponent, reflectivity, refraction
    index, alpha and filter rgb."""

    def __init__(self, n: int):
        self.kind = np.zeros(n, np.int32)
        self.diffuse = np.zeros((n, 3), np.float32)
        self.specular = np.zeros((n, 3), np.float32)
        self.exponent = np.zeros(n, np.int32)
        self.reflectivity = np.zeros(n, np.float32)
        self.refraction = np.zeros(n, np.float32)
        self.alpha = np.zeros(n, np.float32)
        self.filter = np.zeros((n, 3), np.float32)

    def specpow(self) -> np.ndarray:
        """Per-material Phong exponent for the frame renderer (-1 where the
        material is not Phong)."""
        return np.where(self.kind == _lib.RQ_MAT_PHONG, self.exponent, -1).astype(np.int32)


def read_obj(path: str):
    """Reads an OBJ file and its material library: (Mesh, ObjMaterials).
    The mesh's material colours are the table's diffuse colours."""
    h = C.c_void_p()
    check(lib.rq_mesh_read_obj(str(path).encode(), C.byref(h)))
    try:
        nv, nt, nm = C.c_int(), C.c_int(), C.c_int()
        check(lib.rq_mesh_info(h, C.byref(nv), C.byref(nt)))
        check(lib.rq_mesh_material_count(h, C.byref(nm)))
        v = np.zeros((nv.value, 3), np.float32)
        ix = np.zeros((nt.value, 3), np.uint32)
        fm = np.zeros(nt.value, np.uint32)
        check(lib.rq_mesh_copy(h, v.ctypes.data, ix.ctypes.data, fm.ctypes.data))
        m = ObjMaterials(nm.value)
        check(lib.rq_mesh_materials(h, m.kind.ctypes.data, m.diffuse.ctypes.data,
                                    m.specular.ctypes.data, m.exponent.ctypes.data,
                                    m.reflectivity.ctypes.data, m.refraction.ctypes.data,
                                    m.alpha.ctypes.data, m.filter.ctypes.data))
    finally:
        lib.rq_mesh_destroy(h)
    return Mesh(v, ix, fm, m.diffuse.copy()), m


__all__ = ["read_ply", "read_obj", "ObjMaterials", "_lib"]
