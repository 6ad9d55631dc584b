"""DynBVH tree files: the byte stream of DynBVH::saveToFile
(Model/Groups/DynBVH.cc:2479-2501), read by DynBVH::buildFromFile
(DynBVH.cc:2442-2476):

    u32 n_ids | int32 object_ids[n_ids] | u32 n_nodes | BVHNode[n_nodes]

BVHNode is the reference's 32-byte x86-64 record (DynBVH.h:37-52): BBox
(6 float: min xyz, max xyz) at 0, int child at 24, unsigned char axis at 28,
the isLeftCheaper / isLargeSubtree bitfields in bits 0 / 1 of byte 29 and
short children at 30.  The device library parses the same stream in
rq_scene_import_dynbvh; this module is the host-side reader and writer.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

NODE_DTYPE = np.dtype([("bounds", "<f4", (6,)), ("child", "<i4"), ("axis", "u1"),
                       ("bits", "u1"), ("children", "<i2")])
assert NODE_DTYPE.itemsize == 32


@dataclass
class TreeFields:
    bounds: np.ndarray
    child: np.ndarray
    children: np.ndarray
    axis: np.ndarray
    left_cheaper: np.ndarray
    ids: np.ndarray


class TreeFormatError(ValueError):
    pass


def parse_dynbvh_blob(blob: bytes, n_tris: int | None = None) -> TreeFields:
    b = memoryview(blob)
    if len(b) < 8:
        raise TreeFormatError("truncated tree file")
    n_ids = int(np.frombuffer(b[:4], "<u4")[0])
    end_ids = 4 + 4 * n_ids
    if end_ids + 4 > len(b):
        raise TreeFormatError("truncated object_ids")
    ids = np.frombuffer(b[4:end_ids], "<i4").copy()
    n_nodes = int(np.frombuffer(b[end_ids:end_ids + 4], "<u4")[0])
    start = end_ids + 4
    if start + 32 * n_nodes > len(b) or n_nodes == 0:
        raise TreeFormatError("truncated node array")
    nodes = np.frombuffer(b[start:start + 32 * n_nodes], NODE_DTYPE)
    if n_tris is not None:
        if n_ids < n_tris:
            raise TreeFormatError("fewer object ids than triangles")
        ids = ids[:n_tris]
    return TreeFields(nodes["bounds"].copy(), nodes["child"].copy(),
                      nodes["children"].astype(np.int32), nodes["axis"].copy(),
                      (nodes["bits"] & 1).astype(np.uint8), ids)


def write_dynbvh_blob(t: TreeFields) -> bytes:
    n = t.children.shape[0]
    nodes = np.zeros(n, NODE_DTYPE)
    nodes["bounds"] = t.bounds
    nodes["child"] = t.child
    nodes["axis"] = t.axis
    nodes["bits"] = np.asarray(t.left_cheaper, np.uint8) & 1
    nodes["children"] = np.asarray(t.children, np.int16)
    ids = np.asarray(t.ids, "<i4")
    return (np.uint32(ids.shape[0]).tobytes() + ids.tobytes() +
            np.uint32(n).tobytes() + nodes.tobytes())
