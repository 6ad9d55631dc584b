"""Generates the committed golden fixtures from the reference's own code.

    make -f oracle/ref.mk REF=/path/to/rfManta -j8 oracle/_ref/libmanta_ref.so
    python tests/golden/make_golden.py

For each triangle kind (WaldTriangle, KenslerShirleyTriangle) it builds the
small seeded frame scene (level-2 displaced icosphere + 6x6 ground grid, 392
triangles, 48x40 pixels, two point lights) with the reference's Mesh +
DynBVH::rebuild, and records what the reference computes:
  * the tree (field by field) and the DynBVH::saveToFile byte stream;
  * DynBVH::computeCost of that tree;
  * the PinholeCamera basis;
  * DynBVH::intersect results (hit, t, triangle id, u, v) for the frame's
    primary rays, for seeded random closest-hit rays and for seeded random
    any-hit rays;
  * the Raytracer::traceEyeRays frame (RGB, primary t and triangle id) and
    the number of shadow rays HardShadows sent.
It also records DynBVH::computeCost of the reference's own tree for a few
larger seeded scenes (sah_costs.json), the bound for the GPU builder, and a
two-level scene (tiny_instanced.npz): a 12x12 heightfield placed in the
top-level group as a nested DynBVH plus six InstanceT copies of a level-2
displaced icosphere (Phong), with the reference's inner and top-level trees, its
DynBVH::intersect results (closest and AnyHit) for seeded rays and its
Raytracer colours for the 4-spp jittered samples of a 48x40 frame, and
ply_cases.npz: Manta::readPlyFile's vertices, triangles and face materials
for the PLY files the tests write (tests/test_mesh_io.py), and
tree_update.npz: DynBVH::update with its tree rotations over four frames of a
seeded animation (the tree, per-node costs and nextFree after every frame),
and path_stats.npz: KajiyaPathtracer images of the tiny path scene for 16
seeds at 4096 samples per pixel, at depth 4 and at depth 2 with a constant
ambient light (the expectation the path tracer must match),
obj_cases.npz: Manta::ObjGroup's vertices, triangles, face materials and
material table for the OBJ files the tests write, tiny_reflect.npz: the
reference's sample colours of frames with reflective Phong materials, and
tiny_env.npz: frames and path-traced images lit by EyeAmbient over a
LinearBackground.  One flag (--instanced, --ply, --update, --path, --obj,
--reflect, --env) regenerates that fixture alone.
The fixtures pin the CPU restatement (oracle/rq_oracle.c) and the device
path to the reference without needing the reference at test time.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.pyoracle import Reference, Restatement  # noqa: E402
from rfmanta_b200 import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main() -> None:
    ref = Reference()
    restated = Restatement()
    sc = scenes.tiny_frame_scene()
    mesh = sc.mesh
    lo, hi = mesh.bounds()
    pad = 0.25 * (hi - lo)
    o_r, d_r, _, _ = scenes.random_rays(4096, lo - pad, hi + pad, seed=11)
    o_a, d_a, tm_a, _ = scenes.random_rays(4096, lo - pad, hi + pad, seed=12,
                                           anyhit_fraction=1.0)
    for kind, name in ((0, "wald"), (1, "ks")):
        rs = ref.scene(mesh, kind)
        tree = rs.tree()
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "tree.bvh")
            rs.save_blob(path)
            blob = np.frombuffer(open(path, "rb").read(), np.uint8)
        basis = ref.camera_basis(sc.camera)
        org, dir = restated.primary_rays(basis, sc.xres, sc.yres)
        n = org.shape[1]
        prim_q = rs.intersect(org, dir, np.full(n, 1e19, np.float32))
        rnd_q = rs.intersect(o_r, d_r, np.full(o_r.shape[1], 1e19, np.float32))
        any_q = rs.intersect(o_a, d_a, tm_a, anyhit=True)
        img = rs.render(sc, nthreads=1)
        out = dict(
            vertices=mesh.vertices, indices=mesh.indices, face_material=mesh.face_material,
            materials=mesh.materials,
            bounds=tree.bounds, child=tree.child, children=tree.children, axis=tree.axis,
            left_cheaper=tree.left_cheaper, ids=tree.ids, blob=blob,
            node_size=np.int32(ref.lib.mref_node_size()),
            sah_cost=np.float64(rs.sah_cost()), camera_basis=basis,
            xres=np.int32(sc.xres), yres=np.int32(sc.yres),
            lights=np.array([list(l.position) + list(l.color) for l in sc.lights], np.float32),
            ambient=np.asarray(sc.ambient, np.float32),
            background=np.asarray(sc.background, np.float32),
            cam=np.array(list(sc.camera.eye) + list(sc.camera.lookat) + list(sc.camera.up) +
                         [sc.camera.hfov, sc.camera.vfov], np.float32),
            primary_org=org, primary_dir=dir,
            **{f"primary_{k}": v for k, v in prim_q.items()},
            rand_org=o_r, rand_dir=d_r, **{f"rand_{k}": v for k, v in rnd_q.items()},
            any_org=o_a, any_dir=d_a, any_tmax=tm_a, **{f"any_{k}": v for k, v in any_q.items()},
            img_rgb=img["rgb"], img_t=img["t"], img_prim=img["prim"],
            img_shadow_rays=np.int64(img["shadow_rays"]),
        )
        path = os.path.join(OUT, f"tiny_{name}.npz")
        np.savez_compressed(path, **out)
        rs.close()
        print(path, os.path.getsize(path), "bytes")


def write_instanced() -> None:
    ref = Reference()
    restated = Restatement()
    sc = scenes.tiny_coherent_scene()
    inner = [ref.scene(m, 0) for m in sc.inner]
    for r in inner:
        for m, sp in enumerate(sc.specpow):
            if sp >= 0:
                r.set_phong(m, sc.specular[m], int(sp))
    top = ref.instanced(inner, sc.inst_scene, sc.translation, sc.kind)
    lo = np.array([-4.5, -0.5, -4.5], np.float32)
    hi = np.array([4.5, 2.0, 4.5], np.float32)
    o_r, d_r, _, _ = scenes.random_rays(4096, lo, hi, seed=31)
    o_a, d_a, tm_a, _ = scenes.random_rays(4096, lo, hi, seed=32, anyhit_fraction=1.0)
    rnd_q = top.intersect2(o_r, d_r, np.full(o_r.shape[1], 1e19, np.float32))
    any_q = top.intersect2(o_a, d_a, tm_a, anyhit=True)
    px, py = restated.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed)
    img = top.render_coords(sc, px, py)
    out = dict(n_inner=np.int32(len(sc.inner)), inst_scene=sc.inst_scene,
               translation=sc.translation, kind=sc.kind, materials=sc.materials,
               specular=sc.specular, specpow=sc.specpow,
               xres=np.int32(sc.xres), yres=np.int32(sc.yres), spp=np.int32(sc.spp),
               seed=np.int64(sc.seed), sample_px=px, sample_py=py,
               rand_org=o_r, rand_dir=d_r, **{f"rand_{k}": v for k, v in rnd_q.items()},
               any_org=o_a, any_dir=d_a, any_tmax=tm_a,
               **{f"any_{k}": v for k, v in any_q.items()},
               sample_rgb=img["rgb"], sample_t=img["t"], sample_prim=img["prim"],
               shadow_rays=np.int64(img["shadow_rays"]))
    trees = [(f"inner{i}", r.tree()) for i, r in enumerate(inner)] + [("top", top.tree())]
    for name, t in trees:
        for f in ("bounds", "child", "children", "axis", "left_cheaper", "ids"):
            out[f"{name}_{f}"] = getattr(t, f)
    for i, m in enumerate(sc.inner):
        out[f"inner{i}_vertices"] = m.vertices
        out[f"inner{i}_indices"] = m.indices
        out[f"inner{i}_face_material"] = m.face_material
    path = os.path.join(OUT, "tiny_instanced.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


REFLECT = dict(flat_refl=(0.9, 0.8), flat_specpow=(20, 8), instanced_refl=0.6)


def write_reflect() -> None:
    """Reflective Phong (Phong.cc:438-540, Raytracer recursion with the
    default maxDepth 15 and importance cutoff 0.01): the reference's
    per-sample colours of a 40x32, 4-spp frame of the tiny frame scene with
    both materials reflective, and of the tiny two-level scene's frame with
    its Phong spheres reflective (trees: tiny_instanced.npz)."""
    ref = Reference()
    restated = Restatement()
    out = {}
    sc = scenes.tiny_frame_scene(xres=40, yres=32)
    sc.spp, sc.seed = 4, 5
    m = sc.mesh
    rs = ref.scene(m, 0)
    nm = m.materials.shape[0]
    for k in range(nm):
        rs.set_phong(k, np.full(3, 0.4, np.float32), REFLECT["flat_specpow"][k],
                     REFLECT["flat_refl"][k])
    px, py = restated.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed)
    img = rs.render_coords(sc, px, py)
    t = rs.tree()
    for f in ("bounds", "child", "children", "axis", "left_cheaper", "ids"):
        out[f"flat_{f}"] = getattr(t, f)
    out.update(flat_vertices=m.vertices, flat_indices=m.indices,
               flat_face_material=m.face_material, flat_materials=m.materials,
               flat_sample_rgb=img["rgb"], flat_sample_t=img["t"], flat_sample_prim=img["prim"],
               flat_shadow_rays=np.int64(img["shadow_rays"]))
    rs.close()
    sc = scenes.tiny_coherent_scene()
    inner = [ref.scene(mm, 0) for mm in sc.inner]
    for r in inner:
        for k, sp in enumerate(sc.specpow):
            if sp >= 0:
                r.set_phong(k, sc.specular[k], int(sp), REFLECT["instanced_refl"])
    top = ref.instanced(inner, sc.inst_scene, sc.translation, sc.kind)
    px, py = restated.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed)
    img = top.render_coords(sc, px, py)
    out.update(inst_sample_rgb=img["rgb"], inst_sample_t=img["t"],
               inst_sample_prim=img["prim"], inst_shadow_rays=np.int64(img["shadow_rays"]))
    path = os.path.join(OUT, "tiny_reflect.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


# EyeAmbient and LinearBackground (cup = the scene's background colour)
ENVIRONMENT = dict(down=(0.9, 0.3, 0.1), up=(0.2, 1.0, 0.3), path_ambient=(0.3, 0.4, 0.5),
                   path_background=(0.2, 0.3, 0.6), path_depths=(1, 2), seeds=16)


def environment():
    return scenes.Environment(ambient="eye", background="linear",
                              background_down=ENVIRONMENT["down"],
                              background_up=ENVIRONMENT["up"])


def write_environment() -> None:
    """EyeAmbient (Model/AmbientLights/EyeAmbient.cc) and LinearBackground
    (Model/Backgrounds/LinearBackground.cc): the reference's Whitted frame of
    the tiny frame scene (48x40, Raytracer::traceEyeRays), its per-sample
    colours of the 40x32 4-spp reflective Phong frame (materials as in
    tiny_reflect.npz), and KajiyaPathtracer images of the tiny path scene at
    depths 1 and 2 (16 seeds each, 16x12 at 4096 spp, one thread), all with
    both."""
    ref = Reference()
    restated = Restatement()
    env = environment()
    out = {}
    sc = scenes.tiny_frame_scene(xres=48, yres=40)
    sc.environment = env
    m = sc.mesh
    rs = ref.scene(m, 0)
    rs.set_environment(env)
    img = rs.render(sc)
    t = rs.tree()
    for f in ("bounds", "child", "children", "axis", "left_cheaper", "ids"):
        out[f"tree_{f}"] = getattr(t, f)
    out.update(whitted_rgb=img["rgb"], whitted_t=img["t"], whitted_prim=img["prim"],
               whitted_shadow_rays=np.int64(img["shadow_rays"]))
    nm = m.materials.shape[0]
    for k in range(nm):
        rs.set_phong(k, np.full(3, 0.4, np.float32), REFLECT["flat_specpow"][k],
                     REFLECT["flat_refl"][k])
    sc.xres, sc.yres, sc.spp, sc.seed = 40, 32, 4, 5
    px, py = restated.sample_coords(sc.xres, sc.yres, sc.spp, sc.seed)
    img = rs.render_coords(sc, px, py)
    out.update(frame_sample_rgb=img["rgb"], frame_sample_prim=img["prim"],
               frame_shadow_rays=np.int64(img["shadow_rays"]))
    rs.close()
    p = PATH_STATS
    ps = scenes.tiny_path_scene(xres=p["xres"], yres=p["yres"], spp=p["spp"])
    ps.ambient, ps.background = ENVIRONMENT["path_ambient"], ENVIRONMENT["path_background"]
    ps.environment = env
    rp = ref.scene(ps.mesh, 0)
    rp.set_environment(env)
    for depth in ENVIRONMENT["path_depths"]:
        ps.max_depth = depth
        imgs = []
        for s in range(ENVIRONMENT["seeds"]):
            ps.seed = 5000 + 100 * depth + s
            imgs.append(rp.render_path(ps, nthreads=1)["rgb"].reshape(p["yres"], p["xres"], 3))
        out[f"path_images_d{depth}"] = np.array(imgs, np.float32)
    rp.close()
    path = os.path.join(OUT, "tiny_env.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


def write_obj_cases() -> None:
    """Manta::ObjGroup's results for the OBJ files tests/test_mesh_io.py
    writes (vertices, triangles, face materials, material kinds and glm
    values)."""
    import pathlib
    import tempfile
    sys.path.insert(0, os.path.dirname(OUT))
    from test_mesh_io import obj_cases
    ref = Reference()
    out = {"names": np.array([n for n, _, _ in obj_cases()])}
    with tempfile.TemporaryDirectory() as td:
        for name, files, obj in obj_cases():
            d = pathlib.Path(td) / name
            d.mkdir()
            for fn, text in files.items():
                (d / fn).write_text(text)
            v, ix, fm, kind, vals = ref.read_obj(d / obj)
            out[f"{name}_bytes"] = np.frombuffer((d / obj).read_bytes(), np.uint8)
            out[f"{name}_vertices"] = v
            out[f"{name}_indices"] = ix
            out[f"{name}_face_material"] = fm
            out[f"{name}_kind"] = kind
            out[f"{name}_values"] = vals
    path = os.path.join(OUT, "obj_cases.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


def write_ply_cases() -> None:
    import tempfile
    sys.path.insert(0, os.path.dirname(OUT))
    from test_mesh_io import cases, write_ply
    ref = Reference()
    out = {"names": np.array([n for n, _, _ in cases()])}
    with tempfile.TemporaryDirectory() as td:
        for name, kw, transform in cases():
            p = os.path.join(td, name + ".ply")
            write_ply(p, **kw)
            v, ix, fm = ref.read_ply(p, transform)
            out[f"{name}_bytes"] = np.frombuffer(open(p, "rb").read(), np.uint8)
            out[f"{name}_vertices"] = v
            out[f"{name}_indices"] = ix
            out[f"{name}_face_material"] = fm
    path = os.path.join(OUT, "ply_cases.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


def update_cases():
    """Meshes for the animated-mesh update fixture: the tiny frame scene and
    a small one, four frames each of scenes.animated_vertices."""
    return {"tiny": scenes.tiny_frame_scene().mesh,
            "small": scenes.small_frame_scene(level=3, grid=12, xres=8, yres=8).mesh}


UPDATE_FRAMES = 4
DYN_FIELDS = ("bounds", "child", "children", "axis", "left_cheaper", "costs", "ids")


def write_tree_update() -> None:
    """DynBVH::update(0, 1) (tree rotations and leaf re-splits, TREE_ROT 1)
    of the reference's rebuilt tree over four animation frames: the tree,
    per-node costs and nextFree before and after every frame."""
    ref = Reference()
    out = {"names": np.array(list(update_cases()))}
    for name, mesh in update_cases().items():
        rs = ref.scene(mesh, 0)
        v0 = mesh.vertices.copy()
        states = [rs.dyn_tree()]
        for k in range(1, UPDATE_FRAMES + 1):
            v = scenes.animated_vertices(v0, k)
            out[f"{name}_vertices{k}"] = v
            rs.update_vertices(v)
            states.append(rs.dyn_tree())
        for k, st in enumerate(states):
            n = st.next_free
            for f in DYN_FIELDS:
                a = getattr(st, f)
                out[f"{name}_s{k}_{f}"] = a if f == "ids" else a[:n]
            out[f"{name}_s{k}_next_free"] = np.int64(n)
            out[f"{name}_s{k}_cap"] = np.int64(st.cap)
        out[f"{name}_indices"] = mesh.indices
        out[f"{name}_vertices0"] = v0
        rs.close()
    path = os.path.join(OUT, "tree_update.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


PATH_STATS = dict(xres=16, yres=12, spp=4096, seeds=16)
PATH_AMBIENT = (0.3, 0.4, 0.5)


def write_path_stats() -> None:
    """KajiyaPathtracer frames (one thread, so each seed is reproducible) of
    the tiny path scene for several seeds: the reference's estimator that
    the path tracer's images must match in expectation."""
    ref = Reference()
    p = PATH_STATS
    sc = scenes.tiny_path_scene(xres=p["xres"], yres=p["yres"], spp=p["spp"])
    rs = ref.scene(sc.mesh, 0)
    imgs, amb = [], []
    for s in range(p["seeds"]):
        sc.seed = 2000 + s
        sc.ambient = (0.0, 0.0, 0.0)
        imgs.append(rs.render_path(sc, nthreads=1)["rgb"].reshape(p["yres"], p["xres"], 3))
        sc.ambient, sc.max_depth = PATH_AMBIENT, 2  # most paths reach the last bounce
        amb.append(rs.render_path(sc, nthreads=1)["rgb"].reshape(p["yres"], p["xres"], 3))
        sc.max_depth = 4
    rs.close()
    path = os.path.join(OUT, "path_stats.npz")
    np.savez_compressed(path, images=np.array(imgs, np.float32),
                        images_ambient=np.array(amb, np.float32),
                        ambient=np.array(PATH_AMBIENT, np.float32),
                        seed_values=np.arange(2000, 2000 + p["seeds"]),
                        **{k: np.int64(v) for k, v in p.items()})
    print(path, os.path.getsize(path), "bytes")


def sah_scene_makers():
    """Scenes whose reference SAH cost pins the GPU builder (2% bound), as
    name -> generator.  The first three are small; the rest are the
    benchmark scenes at full size: the path-tracing frame (1,212,416
    triangles), the coherent frame's 1024x1024 heightfield (2,097,152), and
    the two largest batched-query scenes (3,276,800 and 5,120,000)."""
    def soup():
        rng = np.random.default_rng(23)
        n = 20000
        c = rng.uniform(-2, 2, (n, 1, 3))
        tri = (c + rng.normal(scale=0.05, size=(n, 3, 3))).reshape(-1, 3).astype(np.float32)
        return scenes.Mesh(tri, np.arange(3 * n, dtype=np.uint32).reshape(-1, 3),
                           np.zeros(n, np.uint32), np.ones((1, 3), np.float32))

    return {
        "small_frame": lambda: scenes.small_frame_scene().mesh,
        "heightfield_256": lambda: scenes.merge(
            [scenes.heightfield(256, 256, seed=21, extent=4.0, y=-1.1),
             scenes.displaced_icosphere(4, seed=22, center=(0.5, 0.0, -0.5), radius=0.6)],
            np.array([[0.5, 0.5, 0.5]], np.float32)),
        "random_soup": soup,
        "path_frame": lambda: scenes.path_scene().mesh,
        "coherent_heightfield": lambda: scenes.coherent_scene().inner[0],
        "query_scene_6": lambda: scenes.query_scene(6),
        "query_scene_7": lambda: scenes.query_scene(7),
    }


def sah_scenes():
    """The small SAH scenes, generated."""
    mk = sah_scene_makers()
    return {k: mk[k]() for k in ("small_frame", "heightfield_256", "random_soup")}


def write_sah_costs() -> None:
    """DynBVH::rebuild (the reference's exact-sweep SAH build) of every SAH
    scene and DynBVH::computeCost of the result (Model/Groups/DynBVH.cc:
    1699-1857, 3389-3416), with the reference's build time."""
    import json
    import time
    ref = Reference()
    costs, secs = {}, {}
    for name, make in sah_scene_makers().items():
        mesh = make()
        t0 = time.perf_counter()
        rs = ref.scene(mesh, 0)
        secs[name] = round(time.perf_counter() - t0, 2)
        costs[name] = rs.sah_cost()
        rs.close()
        print(name, mesh.n_tris, costs[name], secs[name], "s", flush=True)
    path = os.path.join(OUT, "sah_costs.json")
    with open(path, "w") as f:
        json.dump(costs, f, indent=1, sort_keys=True)
    print(path, costs)


if __name__ == "__main__":
    ONE = {"--instanced": write_instanced, "--ply": write_ply_cases,
           "--update": write_tree_update, "--path": write_path_stats,
           "--obj": write_obj_cases, "--reflect": write_reflect, "--env": write_environment,
           "--sah": write_sah_costs}
    chosen = [f for flag, f in ONE.items() if flag in sys.argv]
    if chosen:
        for f in chosen:
            f()
    else:
        main()
        for f in ONE.values():
            f()
