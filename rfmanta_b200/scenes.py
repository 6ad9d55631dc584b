"""Seeded synthetic scenes for the ray-query path.

The reference renders triangle meshes handed to a ``Mesh`` group
(Model/Groups/Mesh.h:27-50): a float vertex array, three vertex indices per
triangle and one material index per triangle.  The generators here produce
exactly those three arrays (float32 / uint32) so that the device path, the
CPU restatement and the reference's own classes all read identical bytes.

Shapes follow the workloads this project measures:
  * displaced icosphere: subdivided icosahedron, vertices pushed along the
    radius by seeded 3-D value noise;
  * ground quad grid: a flat grid of quads split into two triangles each;
  * heightfield: an nx x nz grid whose heights are seeded fractal (fBm)
    2-D value noise.
All arithmetic before the final float32 cast is float64 numpy, which is
IEEE-deterministic, so a seed always yields the same bytes.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Mesh:
    """Triangle soup in the reference's Mesh layout."""

    vertices: np.ndarray  # (V, 3) float32
    indices: np.ndarray  # (T, 3) uint32
    face_material: np.ndarray  # (T,) uint32
    materials: np.ndarray = field(default_factory=lambda: np.zeros((1, 3), np.float32))

    @property
    def n_tris(self) -> int:
        return int(self.indices.shape[0])

    def bounds(self) -> tuple[np.ndarray, np.ndarray]:
        return self.vertices.min(axis=0), self.vertices.max(axis=0)


def merge(meshes: list[Mesh], materials: np.ndarray) -> Mesh:
    """Concatenates meshes; each keeps its own face_material values."""
    verts, idx, mats = [], [], []
    base = 0
    for m in meshes:
        verts.append(m.vertices)
        idx.append(m.indices + np.uint32(base))
        mats.append(m.face_material)
        base += m.vertices.shape[0]
    return Mesh(
        np.ascontiguousarray(np.concatenate(verts).astype(np.float32)),
        np.ascontiguousarray(np.concatenate(idx).astype(np.uint32)),
        np.ascontiguousarray(np.concatenate(mats).astype(np.uint32)),
        np.ascontiguousarray(np.asarray(materials, np.float32).reshape(-1, 3)),
    )


# ---------------------------------------------------------------- noise ----

class ValueNoise:
    """Seeded lattice value noise with smoothstep interpolation."""

    def __init__(self, seed: int, size: int = 256):
        rng = np.random.default_rng(seed)
        self.size = size
        self.perm = rng.permutation(size).astype(np.int64)
        self.vals = rng.random(size)

    def _hash(self, *coords: np.ndarray) -> np.ndarray:
        h = np.zeros_like(coords[0])
        for c in coords:
            h = self.perm[(h + c) % self.size]
        return h

    def noise3(self, p: np.ndarray) -> np.ndarray:
        """p: (N, 3) float64 -> (N,) in [0, 1)."""
        fl = np.floor(p)
        i = fl.astype(np.int64)
        f = p - fl
        s = f * f * (3.0 - 2.0 * f)
        out = np.zeros(p.shape[0])
        for dz in (0, 1):
            wz = s[:, 2] if dz else 1.0 - s[:, 2]
            for dy in (0, 1):
                wy = s[:, 1] if dy else 1.0 - s[:, 1]
                for dx in (0, 1):
                    wx = s[:, 0] if dx else 1.0 - s[:, 0]
                    v = self.vals[self._hash(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)]
                    out += wx * wy * wz * v
        return out

    def noise2(self, p: np.ndarray) -> np.ndarray:
        """p: (N, 2) float64 -> (N,) in [0, 1)."""
        fl = np.floor(p)
        i = fl.astype(np.int64)
        f = p - fl
        s = f * f * (3.0 - 2.0 * f)
        out = np.zeros(p.shape[0])
        for dy in (0, 1):
            wy = s[:, 1] if dy else 1.0 - s[:, 1]
            for dx in (0, 1):
                wx = s[:, 0] if dx else 1.0 - s[:, 0]
                out += wx * wy * self.vals[self._hash(i[:, 0] + dx, i[:, 1] + dy)]
        return out


# ------------------------------------------------------------ primitives ---

def icosphere(level: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4**level triangles (level 6 -> 81,920)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array(
        [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
         [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
         [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(
        [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
         [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
         [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
         [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(level):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mid])
        nf = f.shape[0]
        m01 = base + inv[:nf]
        m12 = base + inv[nf:2 * nf]
        m20 = base + inv[2 * nf:]
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1),
            np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1)])
    return v, f


def displaced_icosphere(level: int = 6, seed: int = 1, amplitude: float = 0.05,
                        frequency: float = 4.0, center=(0.0, 0.0, 0.0),
                        radius: float = 1.0, material: int = 0) -> Mesh:
    """Icosphere with radius r * (1 + amplitude * (2 * noise(freq * p) - 1))."""
    v, f = icosphere(level)
    n = ValueNoise(seed).noise3(v * frequency + 17.0)
    r = radius * (1.0 + amplitude * (2.0 * n - 1.0))
    pos = v * r[:, None] + np.asarray(center, np.float64)
    return Mesh(pos.astype(np.float32), f.astype(np.uint32),
                np.full(f.shape[0], material, np.uint32))


def quad_grid(n_quads_x: int, n_quads_z: int, x0: float, x1: float,
              z0: float, z1: float, heights: np.ndarray | None = None,
              y: float = 0.0, material: int = 0) -> Mesh:
    """(nx x nz) quads, two triangles each; optional per-vertex heights."""
    xs = np.linspace(x0, x1, n_quads_x + 1)
    zs = np.linspace(z0, z1, n_quads_z + 1)
    gx, gz = np.meshgrid(xs, zs, indexing="xy")
    gy = np.full_like(gx, y) if heights is None else y + heights.reshape(gx.shape)
    verts = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1)
    w = n_quads_x + 1
    iz, ix = np.meshgrid(np.arange(n_quads_z), np.arange(n_quads_x), indexing="ij")
    a = (iz * w + ix).ravel()
    b = a + 1
    c = a + w
    d = c + 1
    tris = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)])
    # interleave the two triangles of each quad
    tris = tris.reshape(2, -1, 3).transpose(1, 0, 2).reshape(-1, 3)
    return Mesh(verts.astype(np.float32), tris.astype(np.uint32),
                np.full(tris.shape[0], material, np.uint32))


def fbm_heights(nx: int, nz: int, seed: int, octaves: int = 5,
                amplitude: float = 0.2, base_frequency: float = 4.0) -> np.ndarray:
    """(nz+1, nx+1) fractal value-noise heights in [-amplitude, amplitude]."""
    noise = ValueNoise(seed)
    u = np.linspace(0.0, 1.0, nx + 1)
    w = np.linspace(0.0, 1.0, nz + 1)
    gu, gw = np.meshgrid(u, w, indexing="xy")
    p = np.stack([gu.ravel(), gw.ravel()], 1)
    h = np.zeros(p.shape[0])
    a, fr, norm = 1.0, base_frequency, 0.0
    for o in range(octaves):
        h += a * (2.0 * noise.noise2(p * fr + 31.0 * o) - 1.0)
        norm += a
        a *= 0.5
        fr *= 2.0
    return (amplitude * h / norm).reshape(nz + 1, nx + 1)


def heightfield(nx: int, nz: int, seed: int, extent: float = 4.0,
                octaves: int = 5, amplitude: float = 0.2, y: float = -1.1,
                material: int = 0) -> Mesh:
    """nx x nz heightfield grid (2*nx*nz triangles) of fBm heights."""
    h = fbm_heights(nx, nz, seed, octaves, amplitude)
    e = extent / 2.0
    return quad_grid(nx, nz, -e, e, -e, e, heights=h, y=y, material=material)


# ------------------------------------------------------------ workloads ---

@dataclass
class Camera:
    eye: tuple
    lookat: tuple
    up: tuple
    hfov: float
    vfov: float


@dataclass
class PointLightSpec:
    position: tuple
    color: tuple


@dataclass
class Environment:
    """Ambient light and background beyond the constant forms: ambient
    "constant" (ConstantAmbient) or "eye" (EyeAmbient, Model/AmbientLights/
    EyeAmbient.cc), background "constant" (ConstantBackground) or "linear"
    (LinearBackground, Model/Backgrounds/LinearBackground.cc, with the
    scene's background colour as cup).  The colours stay in the scene's
    `ambient` and `background`."""
    ambient: str = "constant"
    background: str = "constant"
    background_down: tuple = (0.0, 0.0, 0.0)
    background_up: tuple = (0.0, 1.0, 0.0)

    def kinds(self) -> tuple:
        amb = {"constant": 0, "eye": 1}[self.ambient]
        bg = {"constant": 0, "linear": 1}[self.background]
        return amb, bg


@dataclass
class WhittedScene:
    mesh: Mesh
    camera: Camera
    lights: list
    ambient: tuple
    background: tuple
    xres: int
    yres: int
    environment: Environment | None = None


def small_frame_scene(level: int = 6, grid: int = 100, xres: int = 512,
                      yres: int = 512, seed: int = 7) -> WhittedScene:
    """512x512 primary + hard-shadow frame over a displaced icosphere
    (level 6: 81,920 tris, amplitude 0.05, frequency 4) and a 2x2 ground grid
    of 2*grid*grid tris (grid=100: 20,000), one point light at (2,3,2),
    pinhole camera at (0,0,3) looking at the origin, fov 60 degrees."""
    sphere = displaced_icosphere(level, seed=seed, material=0)
    ground = quad_grid(grid, grid, -1.0, 1.0, -1.0, 1.0, y=-1.1, material=1)
    mats = np.array([[0.8, 0.3, 0.2], [0.6, 0.6, 0.6]], np.float32)
    mesh = merge([sphere, ground], mats)
    cam = Camera((0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 60.0, 60.0)
    lights = [PointLightSpec((2.0, 3.0, 2.0), (0.9, 0.9, 0.9))]
    return WhittedScene(mesh, cam, lights, (0.1, 0.1, 0.1), (0.2, 0.3, 0.5), xres, yres)


def tiny_frame_scene(xres: int = 48, yres: int = 40, seed: int = 3) -> WhittedScene:
    """The small-frame layout scaled down (level-2 icosphere, 6x6 grid) for
    committed fixtures."""
    s = small_frame_scene(level=2, grid=6, xres=xres, yres=yres, seed=seed)
    s.lights.append(PointLightSpec((-2.0, 1.5, 2.5), (0.3, 0.35, 0.4)))
    return s


def animated_vertices(v0: np.ndarray, frame: int, amplitude: float = 0.04,
                      jitter: float = 0.01, seed: int = 100) -> np.ndarray:
    """Frame `frame` of a seeded non-rigid animation of a mesh's vertices:
    a travelling sine displacement whose amplitude grows with the frame,
    plus per-vertex noise (the animated-mesh refit workload)."""
    rng = np.random.default_rng(seed + frame)
    w = np.sin(3.0 * v0[:, [1, 2, 0]] + 0.7 * frame).astype(np.float32)
    return np.ascontiguousarray(v0 + np.float32(amplitude * (1 + frame)) * w +
                                rng.normal(scale=jitter, size=v0.shape), np.float32)


def wave_vertices(v0: np.ndarray, frame: int, period: int = 8,
                  amplitude: float = 0.01) -> np.ndarray:
    """Frame `frame` of a periodic non-rigid animation (a travelling sine
    displacement, `period` frames long) for benchmarking animated scenes."""
    ph = np.float32(2.0 * np.pi * (frame % period) / period)
    w = np.sin(np.float32(3.0) * v0[:, [1, 2, 0]] + ph).astype(np.float32)
    return np.ascontiguousarray(v0 + np.float32(amplitude) * w, np.float32)


def random_rays(n: int, lo: np.ndarray, hi: np.ndarray, seed: int,
                anyhit_fraction: float = 0.0):
    """Origins uniform in [lo, hi], directions uniform on the sphere, tmax
    uniform in [0.1, |hi-lo|] (for the any-hit share) or 1e19 (closest)."""
    rng = np.random.default_rng(seed)
    o = lo + (hi - lo) * rng.random((n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    diag = float(np.linalg.norm(hi - lo))
    anyhit = rng.random(n) < anyhit_fraction
    tmax = np.where(anyhit, rng.uniform(0.1, max(diag, 0.1000001), n), 1e19)
    return (np.ascontiguousarray(o.T.astype(np.float32)),
            np.ascontiguousarray(d.T.astype(np.float32)),
            tmax.astype(np.float32), anyhit)


@dataclass
class AreaLightSpec:
    """Parallelogram emitter: anchor + u*v1 + w*v2, u, w in [0, 1)."""

    anchor: tuple
    v1: tuple
    v2: tuple
    color: tuple


@dataclass
class PathScene:
    mesh: Mesh
    camera: Camera
    light: AreaLightSpec
    background: tuple
    xres: int
    yres: int
    spp: int
    max_depth: int
    rr_depth: int
    seed: int = 1
    ambient: tuple = (0.0, 0.0, 0.0)  # ConstantAmbient, added at max_depth
    environment: Environment | None = None


def path_scene(hf_nx: int = 512, hf_nz: int = 1024, n_spheres: int = 32,
               sphere_level: int = 4, xres: int = 1280, yres: int = 720, spp: int = 16,
               max_depth: int = 4, rr_depth: int = 1, seed: int = 17) -> PathScene:
    """Incoherent path-tracing frame: an hf_nx x hf_nz fBm heightfield
    (2*hf_nx*hf_nz triangles, 5 octaves, amplitude 0.2) plus n_spheres
    displaced icospheres at seeded positions on it, one parallelogram area
    light above, diffuse bounces to max_depth with Russian roulette from
    rr_depth on (depth 0 = the camera ray's hit; the reference's
    KajiyaPathtracer applies roulette from depth 1).  Defaults: 1280x720,
    16 spp, depth 4, RR from depth 1,
    1,048,576 + 32 x 5,120 = 1,212,416 triangles."""
    rng = np.random.default_rng(seed)
    ext = 8.0
    parts = [heightfield(hf_nx, hf_nz, seed=seed + 1, extent=ext, y=0.0, material=0)]
    for k in range(n_spheres):
        c = (float(rng.uniform(-3.0, 3.0)), float(rng.uniform(0.3, 0.7)),
             float(rng.uniform(-3.0, 3.0)))
        parts.append(displaced_icosphere(sphere_level, seed=seed + 10 + k, center=c,
                                         radius=float(rng.uniform(0.25, 0.5)),
                                         material=1 + (k % 3)))
    mats = np.array([[0.7, 0.7, 0.65], [0.8, 0.3, 0.2], [0.2, 0.6, 0.3],
                     [0.3, 0.4, 0.8]], np.float32)
    mesh = merge(parts, mats)
    cam = Camera((0.0, 3.5, 7.5), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 60.0,
                 float(2.0 * np.degrees(np.arctan(np.tan(np.radians(30.0)) * yres / xres))))
    light = AreaLightSpec((-1.0, 5.0, -1.0), (2.0, 0.0, 0.0), (0.0, 0.0, 2.0),
                          (30.0, 28.0, 25.0))
    return PathScene(mesh, cam, light, (0.15, 0.2, 0.3), xres, yres, spp, max_depth,
                     rr_depth, seed)


def tiny_path_scene(xres: int = 40, yres: int = 30, spp: int = 4) -> PathScene:
    """The path-tracing layout scaled down for committed checks."""
    return path_scene(hf_nx=16, hf_nz=16, n_spheres=3, sphere_level=2, xres=xres,
                      yres=yres, spp=spp, max_depth=4, rr_depth=1, seed=5)


def sphere_set(n: int, level: int, seed: int, extent: float = 6.0) -> Mesh:
    """n displaced icospheres of the given level at seeded positions."""
    rng = np.random.default_rng(seed)
    v, f = icosphere(level)
    parts = []
    for k in range(n):
        noise = ValueNoise(seed * 1000 + k).noise3(v * 4.0 + 17.0)
        r = float(rng.uniform(0.2, 0.6)) * (1.0 + 0.05 * (2.0 * noise - 1.0))
        c = rng.uniform(-extent / 2, extent / 2, 3)
        parts.append(Mesh((v * r[:, None] + c).astype(np.float32), f.astype(np.uint32),
                          np.zeros(f.shape[0], np.uint32)))
    return merge(parts, np.array([[0.7, 0.7, 0.7]], np.float32))


# (kind, size) of the eight resident scenes of the batched-query workload,
# 10,240 to 5,120,000 triangles
QUERY_SCENE_SPECS = [("spheres", (2, 4)), ("heightfield", 128), ("spheres", (20, 4)),
                     ("heightfield", 384), ("spheres", (12, 6)), ("heightfield", 1024),
                     ("spheres", (40, 6)), ("heightfield", 1600)]


def query_scene(i: int, seed: int = 100) -> Mesh:
    kind, size = QUERY_SCENE_SPECS[i]
    if kind == "spheres":
        return sphere_set(size[0], size[1], seed + i)
    m = heightfield(size, size, seed + i, extent=6.0, y=0.0)
    m.materials = np.array([[0.7, 0.7, 0.7]], np.float32)
    return m


def query_batches(n_batches: int = 64, n_scenes: int = 8, lo: int = 1000,
                  hi: int = 4_000_000, seed: int = 7, scale: float = 1.0):
    """(scene, rays, anyhit) per batch: sizes log-uniform in [lo, hi]
    (times `scale`), scenes uniform, half any-hit."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), n_batches))
    sizes = np.maximum((sizes * scale).astype(np.int64), 1)
    scene = rng.integers(0, n_scenes, n_batches)
    anyhit = rng.random(n_batches) < 0.5
    return [(int(s), int(n), bool(a)) for s, n, a in zip(scene, sizes, anyhit)]


def query_rays_torch(n: int, lo, hi, anyhit: bool, seed: int, device="cuda"):
    """Origins uniform in [lo, hi], directions uniform on the sphere; tmax
    uniform in [0.1, |hi-lo|] for any-hit rays, 1e19 otherwise (torch, on
    the device, from a seeded generator)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    lo_t = torch.tensor(np.asarray(lo, np.float32), device=device).view(3, 1)
    hi_t = torch.tensor(np.asarray(hi, np.float32), device=device).view(3, 1)
    org = lo_t + (hi_t - lo_t) * torch.rand(3, n, generator=g, device=device)
    d = torch.randn(3, n, generator=g, device=device)
    d = d / d.norm(dim=0, keepdim=True)
    diag = float(np.linalg.norm(np.asarray(hi) - np.asarray(lo)))
    if anyhit:
        tmax = 0.1 + (max(diag, 0.1) - 0.1) * torch.rand(n, generator=g, device=device)
    else:
        tmax = torch.full((n,), 1e19, device=device)
    return org.contiguous(), d.contiguous(), tmax.contiguous()


# ------------------------------------------------- two-level frame scene ---

@dataclass
class InstancedFrameScene:
    """A supersampled Whitted frame over a two-level scene: inner meshes
    sharing one material table, instances (inner index, translation, kind:
    0 InstanceT, 1 nested DynBVH)."""
    inner: list
    inst_scene: np.ndarray
    translation: np.ndarray
    kind: np.ndarray
    materials: np.ndarray
    camera: Camera
    lights: list
    ambient: tuple
    background: tuple
    xres: int
    yres: int
    spp: int
    seed: int
    # Phong materials (Model/Materials/Phong.cc without reflection): specular
    # colour per material and exponent, specpow < 0 = Lambertian
    specular: np.ndarray | None = None
    specpow: np.ndarray | None = None
    environment: Environment | None = None

    @property
    def n_tris(self) -> int:
        return int(sum(self.inner[i].n_tris for i in self.inst_scene))


def coherent_scene(hf_n: int = 1024, n_instances: int = 64, sphere_level: int = 6,
                   xres: int = 1920, yres: int = 1080, spp: int = 4,
                   seed: int = 23) -> InstancedFrameScene:
    """Large coherent frame: an hf_n x hf_n fBm heightfield (2*hf_n^2
    triangles, 5 octaves, amplitude 0.2, Lambertian) placed in the top-level
    group as a nested DynBVH, plus n_instances InstanceT copies of one
    displaced icosphere (level 6: 81,920 triangles, amplitude 0.05,
    frequency 4; Phong, specular 0.6, exponent 32) at seeded uniform
    positions above it; two point lights, spp stratified jittered samples
    per pixel.  Defaults: 1920x1080x4,
    2,097,152 + 64 x 81,920 triangles."""
    rng = np.random.default_rng(seed)
    ext = 8.0
    hf = heightfield(hf_n, hf_n, seed=seed + 1, extent=ext, y=0.0, material=0)
    sphere = displaced_icosphere(sphere_level, seed=seed + 2, radius=0.35, material=1)
    pos = np.stack([rng.uniform(-3.5, 3.5, n_instances), rng.uniform(0.45, 0.9, n_instances),
                    rng.uniform(-3.5, 3.5, n_instances)], 1).astype(np.float32)
    inst_scene = np.concatenate([[0], np.ones(n_instances)]).astype(np.int32)
    translation = np.concatenate([np.zeros((1, 3), np.float32), pos]).astype(np.float32)
    kind = np.concatenate([[1], np.zeros(n_instances)]).astype(np.int32)
    mats = np.array([[0.7, 0.7, 0.65], [0.8, 0.3, 0.2]], np.float32)
    hf.materials = mats
    sphere.materials = mats
    cam = Camera((0.0, 4.0, 8.5), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 60.0,
                 float(2.0 * np.degrees(np.arctan(np.tan(np.radians(30.0)) * yres / xres))))
    lights = [PointLightSpec((3.0, 6.0, 4.0), (0.8, 0.8, 0.75)),
              PointLightSpec((-4.0, 5.0, -2.0), (0.35, 0.4, 0.5))]
    specular = np.array([[0.0, 0.0, 0.0], [0.6, 0.6, 0.6]], np.float32)
    specpow = np.array([-1, 32], np.int32)
    return InstancedFrameScene([hf, sphere], inst_scene, translation, kind, mats, cam, lights,
                               (0.08, 0.08, 0.1), (0.2, 0.3, 0.5), xres, yres, spp, seed,
                               specular, specpow)


def tiny_coherent_scene(xres: int = 48, yres: int = 40, spp: int = 4,
                        n_instances: int = 6) -> InstancedFrameScene:
    """The coherent-frame layout scaled down for committed checks."""
    return coherent_scene(hf_n=12, n_instances=n_instances, sphere_level=2, xres=xres,
                          yres=yres, spp=spp, seed=9)
