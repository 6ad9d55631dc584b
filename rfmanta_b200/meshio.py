"""Mesh files through the C ABI: PLY (rq_mesh_read_ply, the reader of
Manta::readPlyFile, Model/Readers/PlyReader.cc) into a scenes.Mesh ready for
GpuDynBVH.setGroup."""
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


__all__ = ["read_ply", "_lib"]
