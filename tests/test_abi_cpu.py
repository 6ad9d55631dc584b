"""The C-ABI library loads and exports every entry point the header
declares; argument errors come back as status codes (no GPU needed)."""
import ctypes as C

import numpy as np


def test_exports_every_declared_symbol():
    from rfmanta_b200 import _lib
    declared = _lib.declared_symbols()
    assert len(declared) >= 14
    for name in declared:
        assert hasattr(_lib.lib, name), name


def test_version_string():
    from rfmanta_b200 import _lib
    assert _lib.lib.rq_version().decode().startswith("rfmanta_b200")


def test_argument_errors_are_status_codes():
    from rfmanta_b200 import _lib
    L = _lib.lib
    h = C.c_void_p()
    assert L.rq_scene_create(None, 0, None, 0, None, 0, 0, C.byref(h)) == _lib.RQ_ERR_ARG
    assert b"empty" in L.rq_last_error()
    v = np.zeros((3, 3), np.float32)
    ix = np.array([[0, 1, 5]], np.uint32)  # index out of range
    assert L.rq_scene_create(v.ctypes.data, 3, ix.ctypes.data, 1, None, 0, 0,
                             C.byref(h)) == _lib.RQ_ERR_ARG
    ix = np.array([[0, 1, 2]], np.uint32)
    assert L.rq_scene_create(v.ctypes.data, 3, ix.ctypes.data, 1, None, 7, 0,
                             C.byref(h)) == _lib.RQ_ERR_ARG
    assert L.rq_trace(None, 4, None, None, None, 0, None, None, None, None) == _lib.RQ_ERR_ARG
    assert L.rq_scene_sah_cost(None, None) == _lib.RQ_ERR_ARG


def test_treeio_roundtrip(golden):
    from rfmanta_b200.treeio import parse_dynbvh_blob, write_dynbvh_blob
    _, g = golden
    blob = g["blob"].tobytes()
    t = parse_dynbvh_blob(blob)
    assert write_dynbvh_blob(t)[:4 + 4 * len(t.ids)] == blob[:4 + 4 * len(t.ids)]
    t2 = parse_dynbvh_blob(write_dynbvh_blob(t))
    for f in ("bounds", "child", "children", "axis", "left_cheaper", "ids"):
        assert np.array_equal(getattr(t, f), getattr(t2, f))


def test_camera_basis_matches_reference(golden):
    """rq_camera_basis (host-only) equals the reference PinholeCamera basis."""
    from rfmanta_b200.dynbvh import camera_basis
    from rfmanta_b200.scenes import Camera
    _, g = golden
    c = g["cam"]
    cam = Camera(tuple(c[0:3]), tuple(c[3:6]), tuple(c[6:9]), float(c[9]), float(c[10]))
    assert np.array_equal(camera_basis(cam).view(np.uint32),
                          g["camera_basis"].view(np.uint32))
