"""PLY reading (rq_mesh_read_ply) against the reference's own reader,
Manta::readPlyFile (Model/Readers/PlyReader.cc) over its vendored rply
parser, compiled from the reference sources: vertices (bit for bit),
triangle indices and face materials must agree on every case, including the
reference's quirks (degenerate-triangle removal by swap-with-last, the last
vertex lost when no face is read, the transform's float order).  Cases are
pinned twice: by the committed fixture tests/golden/ply_cases.npz (the
reference's outputs for these files) and, where the reference library is
built, live.

The reference's reader builds a triangle fan from every polygon but sizes
its triangle array by the number of faces (PlyReader.cc:218-228), so a file
with quads or larger polygons overruns that array; its parity cases are
therefore triangle meshes, and polygon fans are checked against the fan rule
itself (test_polygon_fans)."""
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN

TYPES = {"char": "b", "uchar": "B", "short": "h", "ushort": "H", "int": "i", "uint": "I",
         "float": "f", "double": "d"}


def write_ply(path, fmt, vprops, verts, faces, count_type="uchar", index_type="int",
              face_extra=None, face_prop="vertex_indices", elements_order=("vertex", "face")):
    """vprops: [(type, name)], verts: rows of values; faces: lists of
    indices; face_extra: (type, name, values) added after the list."""
    hdr = ["ply", f"format {fmt} 1.0", "comment written by the rfmanta_b200 tests"]
    for el in elements_order:
        if el == "vertex":
            hdr.append(f"element vertex {len(verts)}")
            hdr += [f"property {t} {n}" for t, n in vprops]
        else:
            hdr.append(f"element face {len(faces)}")
            hdr.append(f"property list {count_type} {index_type} {face_prop}")
            if face_extra:
                hdr.append(f"property {face_extra[0]} {face_extra[1]}")
    hdr.append("end_header")
    body = b""
    if fmt == "ascii":
        lines = []
        for el in elements_order:
            if el == "vertex":
                for row in verts:
                    lines.append(" ".join(repr(float(x)) if t in ("float", "double") else str(int(x))
                                          for (t, _), x in zip(vprops, row)))
            else:
                for k, f in enumerate(faces):
                    s = " ".join([str(len(f))] + [str(i) for i in f])
                    if face_extra:
                        s += " " + str(face_extra[2][k])
                    lines.append(s)
        body = ("\n".join(lines) + "\n").encode()
    else:
        e = "<" if fmt == "binary_little_endian" else ">"
        chunks = []
        for el in elements_order:
            if el == "vertex":
                for row in verts:
                    for (t, _), x in zip(vprops, row):
                        chunks.append(struct.pack(e + TYPES[t], x if t in ("float", "double") else int(x)))
            else:
                for k, f in enumerate(faces):
                    chunks.append(struct.pack(e + TYPES[count_type], len(f)))
                    chunks.append(struct.pack(e + TYPES[index_type] * len(f), *f))
                    if face_extra:
                        chunks.append(struct.pack(e + TYPES[face_extra[0]], face_extra[2][k]))
        body = b"".join(chunks)
    with open(path, "wb") as fh:
        fh.write(("\n".join(hdr) + "\n").encode() + body)


def _tris_of(quads):
    return [t for q in quads for t in ([q[0], q[1], q[2]], [q[0], q[2], q[3]])]


def cases():
    """(name, writer kwargs, transform) of the parity cases (triangles)."""
    rng = np.random.default_rng(7)
    grid = [(x, y, float(np.sin(x + y))) for y in range(4) for x in range(4)]
    quads = [[y * 4 + x, y * 4 + x + 1, (y + 1) * 4 + x + 1, (y + 1) * 4 + x]
             for y in range(3) for x in range(3)]
    pts = rng.normal(size=(30, 3)).round(3).tolist()
    tris = [[int(i) for i in rng.choice(30, size=3, replace=False)] for _ in range(40)]
    # degenerate: repeated index, collinear points, the last triangle degenerate
    line = [(0, 0, 0), (1, 1, 1), (2, 2, 2), (0, 1, 0), (0, -0.0, 1)]
    degen = [[0, 1, 2], [0, 0, 3], [0, 3, 4], [1, 1, 1], [2, 1, 3], [3, 0, 4], [1, 2, 0]]
    fxyz = [("float", "x"), ("float", "y"), ("float", "z")]
    rot = np.array([[0.6, -0.8, 0.0, 1.25], [0.8, 0.6, 0.0, -3.5], [0.0, 0.0, 1.0, 0.1]],
                   np.float32)
    out = [
        ("ascii_grid", dict(fmt="ascii", vprops=fxyz, verts=grid, faces=_tris_of(quads)), None),
        ("le_triangles", dict(fmt="binary_little_endian", vprops=fxyz, verts=pts, faces=tris),
         None),
        ("be_triangles_uint_index", dict(fmt="binary_big_endian", vprops=fxyz, verts=pts,
                                         faces=tris, count_type="uint", index_type="uint"), None),
        ("ascii_double_extra_props", dict(
            fmt="ascii", vprops=[("double", "x"), ("float", "nx"), ("double", "y"),
                                 ("double", "z"), ("uchar", "diffuse_red")],
            verts=[(a, 0.5, b, c, 200) for a, b, c in pts], faces=tris,
            face_extra=("uchar", "flags", [k % 3 for k in range(len(tris))])), None),
        ("le_int_coords_transform", dict(
            fmt="binary_little_endian", vprops=[("int", "x"), ("short", "y"), ("int", "z")],
            verts=[(int(a * 100), int(b * 100), int(c * 100)) for a, b, c in pts],
            faces=tris), rot),
        ("ascii_degenerate", dict(fmt="ascii", vprops=fxyz, verts=line, faces=degen), None),
        ("le_degenerate_transform", dict(fmt="binary_little_endian", vprops=fxyz, verts=line,
                                         faces=degen), rot),
        ("ascii_no_faces", dict(fmt="ascii", vprops=fxyz, verts=grid, faces=[]), None),
        ("ascii_vertex_index_name", dict(fmt="ascii", vprops=fxyz, verts=grid,
                                         faces=_tris_of(quads), face_prop="vertex_index"), None),
    ]
    return out


def _product(path, transform):
    from rfmanta_b200.meshio import read_ply
    m = read_ply(path, transform)
    return m.vertices, m.indices, m.face_material


def _same(a, b):
    va, ia, fa = a
    vb, ib, fb = b
    assert va.shape == vb.shape, (va.shape, vb.shape)
    assert np.array_equal(va.view(np.uint32), vb.view(np.uint32)), "vertices differ"
    assert np.array_equal(ia, ib), "indices differ"
    assert np.array_equal(fa, fb), "face materials differ"


def test_fixture_cases(tmp_path):
    z = np.load(os.path.join(GOLDEN, "ply_cases.npz"))
    names = [n for n, _, _ in cases()]
    assert sorted(str(x) for x in z["names"]) == sorted(names)
    for name, kw, transform in cases():
        p = tmp_path / f"{name}.ply"
        write_ply(p, **kw)
        assert p.read_bytes() == bytes(z[f"{name}_bytes"]), f"{name}: writer changed"
        got = _product(p, transform)
        exp = (z[f"{name}_vertices"], z[f"{name}_indices"], z[f"{name}_face_material"])
        _same(got, exp)


def test_live_reference(tmp_path):
    from oracle.pyoracle import Reference
    if not Reference.available():
        pytest.skip("reference library not built")
    ref = Reference()
    for name, kw, transform in cases():
        p = tmp_path / f"{name}.ply"
        write_ply(p, **kw)
        exp = ref.read_ply(p, transform)
        assert exp is not None, name
        _same(_product(p, transform), exp)


def test_quirks_are_the_references(tmp_path):
    """The behaviours the parity cases pin, stated directly."""
    for name, kw, transform in cases():
        p = tmp_path / f"{name}.ply"
        write_ply(p, **kw)
        v, ix, fm = _product(p, transform)
        if name in ("ascii_no_faces", "ascii_vertex_index_name"):
            assert v.shape[0] == len(kw["verts"]) - 1 and ix.shape[0] == 0
        if name == "ascii_grid":
            assert ix.shape[0] == len(kw["faces"]) and np.all(fm == 0)
        if name == "ascii_degenerate":
            # [0,1,2] and [1,2,0] collinear, [0,0,3] and [1,1,1] repeated:
            # four removed, each slot refilled from the end and re-tested
            assert ix.shape[0] == len(kw["faces"]) - 4


def test_polygon_fans(tmp_path):
    """Polygons become fans (first, previous, current), in file order."""
    rng = np.random.default_rng(9)
    pts = rng.normal(size=(40, 3)).astype(np.float32)
    polys = [[int(i) for i in rng.choice(40, size=int(rng.integers(3, 8)), replace=False)]
             for _ in range(30)]
    p = tmp_path / "poly.ply"
    write_ply(p, "binary_little_endian", [("float", "x"), ("float", "y"), ("float", "z")],
              pts.tolist(), polys)
    v, ix, fm = _product(p, None)
    fan = [[f[0], f[k - 1], f[k]] for f in polys for k in range(2, len(f))]
    assert np.array_equal(v, pts)
    assert np.array_equal(ix, np.array(fan, np.uint32))  # random points: none degenerate


def test_errors(tmp_path):
    from rfmanta_b200._lib import RQ_ERR_FORMAT, RQ_ERR_NOTFOUND, RQError
    from rfmanta_b200.meshio import read_ply
    with pytest.raises(RQError) as e:
        read_ply(tmp_path / "missing.ply")
    assert e.value.code == RQ_ERR_NOTFOUND
    name, kw, _ = cases()[1]
    p = tmp_path / "t.ply"
    write_ply(p, **kw)
    data = p.read_bytes()
    (tmp_path / "cut.ply").write_bytes(data[:-7])
    with pytest.raises(RQError) as e:
        read_ply(tmp_path / "cut.ply")
    assert e.value.code == RQ_ERR_FORMAT
    (tmp_path / "bad.ply").write_bytes(b"ply\nformat ascii 1.0\nelement vertex 1\n"
                                       b"property float x\nend_header\nnotanumber\n")
    with pytest.raises(RQError):
        read_ply(tmp_path / "bad.ply")


@pytest.mark.gpu
def test_ply_mesh_traces(tmp_path):
    """A mesh read from PLY goes straight into a device scene."""
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH, RayBatch
    from rfmanta_b200.meshio import read_ply
    sph = scenes.displaced_icosphere(3, seed=4)
    p = tmp_path / "sphere.ply"
    write_ply(p, "binary_little_endian", [("float", "x"), ("float", "y"), ("float", "z")],
              sph.vertices.tolist(), sph.indices.tolist())
    m = read_ply(p)
    assert np.array_equal(m.vertices, sph.vertices) and np.array_equal(m.indices, sph.indices)
    bvh = GpuDynBVH()
    bvh.setGroup(m)
    bvh.rebuild()
    o = np.zeros((3, 4), np.float32)
    o[0] = [0.1, -0.2, 0.05, 0.3]
    o[1] = [0.05, 0.1, -0.3, -0.1]
    o[2] = 3.0
    d = np.zeros((3, 4), np.float32)
    d[2] = -1.0
    r = RayBatch(o, d)
    bvh.intersect(r)
    assert np.all(r.hitPrim >= 0)


# ----------------------------------------------------------------- OBJ ---

MTL_MAIN = """# materials
newmtl red
Kd 0.9 0.1 0.1
Ka 0.1 0.1 0.1
illum 2
newmtl shiny
Kd 0.2 0.3 0.4
Ks 0.5 0.5 0.5
Ns 32.7
map_Kd -s 2 2 tex.png
newmtl glass
Ni 1.5
newmtl fog
d 0.5
newmtl tinted
Tf 0.9 1 1
newmtl clear
Tr 1
Ns 8
newmtl two words
Kd 0.25 0.5 0.75
"""


def obj_cases():
    """(name, {file name: text}, obj file) of the OBJ parity cases."""
    rng = np.random.default_rng(11)
    pts = rng.normal(size=(24, 3)).round(4)
    vlines = "".join(f"v {x!r} {y!r} {z!r}\n" for x, y, z in pts.tolist())
    faces = [[int(i) + 1 for i in rng.choice(24, size=int(rng.integers(3, 7)), replace=False)]
             for _ in range(30)]
    flines = "".join("f " + " ".join(str(i) for i in f) + "\n" for f in faces)
    basic = ("# groups, materials, fans, relative indices, v/t/n forms\n"
             "mtllib main.mtl\n" + vlines +
             "vt 0 0\nvt 1 0\nvt 1 1\nvn 0 0 1\nvn 0 1 0\n"
             "g first\nusemtl red\nf 1 2 3 4\n"
             "g second\nusemtl shiny\nf 1/1/1 2/2/2 5/3/1\nf -1 -2 -3\n"
             "usemtl unknown\nf 2//1 3//2 6//1 7//2\n"
             "g first\nf 3 4 6\nusemtl glass\nf 4 1 6\n"
             "o third\nusemtl fog\nf 1/1 3/2 5/3\n"
             "s 1\nl 1 2\ng fourth\nusemtl tinted\nf 7 8 9\nusemtl clear\nf 9 10 11\n"
             "usemtl x two\nf 10 11 12\n")
    plain = "# no material library, no groups\n" + vlines + flines
    grid = "".join(f"v {x} {y} 0\n" for y in range(4) for x in range(4))
    degen = ("mtllib main.mtl\n" + grid + "v 0 0 0\n"
             "usemtl red\nf 1 2 3\nf 1 1 5\nf 1 2 5\n"  # collinear / repeated
             "g quad\nf 1 2 6 5\nf 17 1 2\nf 5 6 7 8\nf 2 3 4\n")
    mtl_pre = "Kd 0.3 0.3 0.3\nnewmtl only\nKd 0.6 0.7 0.8\n"
    defaults = ("mtllib pre.mtl\n" + grid + "g a\nf 1 2 6\nusemtl NO_ASSIGNED_MATERIAL\n"
                "f 2 3 7\ng b\nusemtl only\nf 3 4 8\ng c\nf 5 6 10\n")
    two_libs = ("mtllib pre.mtl\nmtllib main.mtl\n" + grid +
                "usemtl only\nf 1 2 6\nusemtl red\nf 2 3 7\n")
    return [
        ("basic", {"main.mtl": MTL_MAIN, "basic.obj": basic}, "basic.obj"),
        ("plain", {"plain.obj": plain}, "plain.obj"),
        ("degenerate", {"main.mtl": MTL_MAIN, "degen.obj": degen}, "degen.obj"),
        ("defaults", {"pre.mtl": mtl_pre, "defaults.obj": defaults}, "defaults.obj"),
        ("two_libs", {"pre.mtl": mtl_pre, "main.mtl": MTL_MAIN, "two.obj": two_libs}, "two.obj"),
    ]


def _write_case(d, files):
    for name, text in files.items():
        (d / name).write_text(text)


def _obj_product(path):
    from rfmanta_b200.meshio import read_obj
    m, mats = read_obj(path)
    vals = np.concatenate([mats.diffuse, mats.specular, mats.exponent[:, None].astype(np.float32),
                           mats.refraction[:, None], mats.alpha[:, None], mats.filter,
                           mats.reflectivity[:, None]], axis=1)
    return m.vertices, m.indices, m.face_material, mats.kind, vals, mats


def _obj_same(got, exp, name):
    v, ix, fm, kind, vals, mats = got
    ev, eix, efm, ekind, evals = exp
    assert np.array_equal(v.view(np.uint32), np.ascontiguousarray(ev, np.float32).view(np.uint32)), name
    assert np.array_equal(ix, eix), f"{name}: triangles differ"
    assert np.array_equal(fm, efm), f"{name}: face materials differ"
    assert np.array_equal(kind, ekind), f"{name}: material kinds differ"
    # the reference reports glm's values for library materials (entries 1..)
    ev = np.array(evals, np.float32)
    if len(kind) > 1:
        assert np.array_equal(mats.diffuse[1:], ev[1:, 0:3]), name
        assert np.array_equal(mats.specular[1:], ev[1:, 3:6]), name
        assert np.array_equal(mats.exponent[1:], ev[1:, 6].astype(np.int32)), name
        assert np.array_equal(mats.refraction[1:], ev[1:, 7]), name
        assert np.array_equal(mats.alpha[1:], ev[1:, 8]), name
        assert np.array_equal(mats.filter[1:], ev[1:, 9:12]), name
        assert np.array_equal(mats.reflectivity[1:], ev[1:, 12]), name


def test_obj_fixture_cases(tmp_path):
    z = np.load(os.path.join(GOLDEN, "obj_cases.npz"))
    names = [n for n, _, _ in obj_cases()]
    assert sorted(str(x) for x in z["names"]) == sorted(names)
    for name, files, obj in obj_cases():
        d = tmp_path / name
        d.mkdir()
        _write_case(d, files)
        assert (d / obj).read_bytes() == bytes(z[f"{name}_bytes"]), f"{name}: writer changed"
        exp = tuple(z[f"{name}_{k}"] for k in ("vertices", "indices", "face_material", "kind",
                                                "values"))
        _obj_same(_obj_product(d / obj), exp, name)


def test_obj_live_reference(tmp_path):
    from oracle.pyoracle import Reference
    if not Reference.available():
        pytest.skip("reference library not built")
    ref = Reference()
    for name, files, obj in obj_cases():
        d = tmp_path / name
        d.mkdir()
        _write_case(d, files)
        exp = ref.read_obj(d / obj)
        assert exp is not None, name
        _obj_same(_obj_product(d / obj), exp, name)


def test_obj_rules(tmp_path):
    """The behaviours the parity cases pin, stated directly."""
    from rfmanta_b200._lib import RQ_MAT_DEFAULT, RQ_MAT_PHONG
    cases = {n: (f, o) for n, f, o in obj_cases()}
    d = tmp_path / "basic"
    d.mkdir()
    _write_case(d, cases["basic"][0])
    v, ix, fm, kind, vals, mats = _obj_product(d / "basic.obj")
    # entry 0 ObjGroup's default, 1 glm's NO_ASSIGNED_MATERIAL, then the
    # library in order: red, shiny, glass, fog, tinted, clear, words
    assert kind[0] == RQ_MAT_DEFAULT
    assert list(kind[1:]) == [0, 0, 1, 2, 3, 3, 1, 0]  # "clear": Tr 1 is white, Ns 8
    assert mats.exponent[3] == 32  # int(Ns 32.7)
    # "newmtl two words" names the material "words" and "usemtl x two"
    # selects "two" (each takes its line's second word), which the library
    # lacks, so glm's material 0: the newest group's face has material 1
    assert fm[0] == 1
    assert np.array_equal(mats.diffuse[8], np.array([0.25, 0.5, 0.75], np.float32))
    d = tmp_path / "plain"
    d.mkdir()
    _write_case(d, cases["plain"][0])
    v, ix, fm, kind, vals, mats = _obj_product(d / "plain.obj")
    assert np.all(fm == 0) and list(kind) == [RQ_MAT_DEFAULT]


def test_obj_errors(tmp_path):
    from rfmanta_b200._lib import RQ_ERR_FORMAT, RQ_ERR_NOTFOUND, RQError
    from rfmanta_b200.meshio import read_obj
    with pytest.raises(RQError) as e:
        read_obj(tmp_path / "missing.obj")
    assert e.value.code == RQ_ERR_NOTFOUND
    (tmp_path / "nolib.obj").write_text("mtllib nothere.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    with pytest.raises(RQError) as e:
        read_obj(tmp_path / "nolib.obj")
    assert e.value.code == RQ_ERR_NOTFOUND
    (tmp_path / "range.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n")
    with pytest.raises(RQError) as e:
        read_obj(tmp_path / "range.obj")
    assert e.value.code == RQ_ERR_FORMAT
    (tmp_path / "w.obj").write_text("v 0 0 0 1\nv 1 0 0 1\nv 0 1 0 1\nf 1 2 3\n")
    with pytest.raises(RQError) as e:
        read_obj(tmp_path / "w.obj")
    assert e.value.code == RQ_ERR_FORMAT


@pytest.mark.gpu
def test_obj_mesh_renders(tmp_path, restatement):
    """An OBJ mesh with its material table goes into a device scene and a
    supersampled frame (Phong entries with their exponents) equals the
    restatement's."""
    from oracle.pyoracle import Tree
    from rfmanta_b200 import scenes
    from rfmanta_b200.dynbvh import GpuDynBVH
    from rfmanta_b200.meshio import read_obj
    from rfmanta_b200.treeio import parse_dynbvh_blob
    name, files, obj = obj_cases()[0]
    _write_case(tmp_path, files)
    mesh, mats = read_obj(tmp_path / obj)
    bvh = GpuDynBVH()
    bvh.setGroup(mesh)
    bvh.rebuild()
    sc = scenes.tiny_frame_scene(xres=32, yres=24)
    sc.mesh = mesh
    sc.spp, sc.seed = 4, 7
    sc.specpow = mats.specpow()
    sc.specular = mats.specular
    sc.camera = scenes.Camera(eye=(0.5, -2.5, 3.0), lookat=(0.0, 0.0, 0.0), up=(0.0, 0.0, 1.0),
                              hfov=60.0, vfov=45.0)
    out = bvh.render_frame(sc, mesh.materials)
    f = parse_dynbvh_blob(bvh.exportBlob(), mesh.n_tris)
    W = restatement.world(Tree(f.bounds, f.child, f.children, f.axis, f.left_cheaper, f.ids),
                          mesh)
    exp = restatement.render_frame(W, sc, mesh.materials, specular=mats.specular,
                                   specpow=sc.specpow)
    assert out["shadow_rays"] == exp["shadow_rays"]
    assert np.array_equal(out["rgb"].view(np.uint32), exp["rgb"].view(np.uint32))
    assert np.count_nonzero(out["rgb"].sum(1)) > 0
