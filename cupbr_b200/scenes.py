"""Scene descriptions and the seeded synthetic scenes the benchmarks use.

A SceneDesc is plain data in cupbr's scene vocabulary (lib/include/Scene/
Scene.h:15-34: geometry objects with one Material each, Lights, an optional
lat-long environment map and the scene Volume).  It can be committed to the
GPU (`build()`), written as cupbr scene XML + OBJ files (`to_xml()`) and
flattened for the CPU checkers (`flat()`).

Synthetic scenes (seeded, deterministic):
  cornell_box()          512x512-class Cornell box: 5 unit quads, two boxes
                         rotated about y (12 triangles each), 0.25x0.25
                         ceiling area light with radiance (17, 12, 4)
  heightfield_spheres()  fBm heightfield (1024x1024 vertex grid, first 1M
                         triangles in row-major order) in 32x32-quad MESH
                         chunks + 200 subdivision-4 icospheres, materials
                         drawn from {Lambert, GGX, dielectric}, procedural
                         2048x1024 sky; 2,024,000 triangles in total
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Optional

import numpy as np

SPHERE, PLANE, QUAD, TRIANGLE, MESH = 0, 1, 2, 3, 4
LAMBERT, PHONG, MIRROR, GLASS, GGX, VOLUME = 0, 1, 2, 3, 4, 5
POINT, AREA = 0, 1
_MAT_NAMES = ["LAMBERT", "PHONG", "MIRROR", "GLASS", "GGX", "VOLUME"]
_GEO_NAMES = ["SPHERE", "PLANE", "QUAD", "TRIANGLE", "MESH"]


@dataclasses.dataclass
class MaterialDesc:
    """Material.h:34-42 / Volume.h:17-20 defaults."""
    type: int = LAMBERT
    albedo_e: tuple = (0.0, 0.0, 0.0)
    albedo_d: tuple = (1.0, 1.0, 1.0)
    albedo_s: tuple = (0.0, 0.0, 0.0)
    shininess: float = 128.0 * 0.4
    roughness: float = 1.0
    eta: float = 1.5
    sigma_s: tuple = (1.0, 1.0, 1.0)
    sigma_a: tuple = (1.0, 1.0, 1.0)
    g: float = 0.0
    interface_glass: int = 0

    def flat(self) -> np.ndarray:
        """21 floats: the checker layout (oracle/oracle_capi.cpp)."""
        return np.array([self.type, *self.albedo_e, *self.albedo_d, *self.albedo_s, self.shininess,
                         np.float32(self.roughness), self.eta, *self.sigma_s, *self.sigma_a, self.g,
                         self.interface_glass], dtype=np.float32)


@dataclasses.dataclass
class LightDesc:
    type: int = AREA
    position: tuple = (0.0, 0.0, 0.0)
    intensity: tuple = (0.0, 0.0, 0.0)
    radiance: tuple = (0.0, 0.0, 0.0)
    half_extend1: tuple = (0.0, 0.0, 0.0)
    half_extend2: tuple = (0.0, 0.0, 0.0)

    def flat(self) -> np.ndarray:
        return np.array([self.type, *self.position, *self.intensity, *self.radiance, *self.half_extend1,
                         *self.half_extend2], dtype=np.float32)


@dataclasses.dataclass
class ObjectDesc:
    type: int
    material: MaterialDesc
    p0: tuple = (0.0, 0.0, 0.0)
    p1: tuple = (0.0, 0.0, 0.0)
    p2: tuple = (0.0, 0.0, 0.0)
    p3: tuple = (0.0, 0.0, 0.0)
    radius: float = 0.0
    vertices: Optional[np.ndarray] = None   # (nv, 3) float32, object space (MESH) or world (TRIANGLE)
    indices: Optional[np.ndarray] = None    # (nt, 3) uint32
    position: tuple = (0.0, 0.0, 0.0)       # MESH transform: scale * v + position (ObjLoader.cpp:37)
    scale: tuple = (1.0, 1.0, 1.0)
    # albedo-texture binding (origin, u_axis, v_axis): planar projection of
    # the scene's texture (cupbr_scene_set_object_texture); None: untextured
    tex_frame: Optional[tuple] = None

    def world_vertices(self) -> np.ndarray:
        v = np.asarray(self.vertices, dtype=np.float32)
        s = np.asarray(self.scale, dtype=np.float32)
        p = np.asarray(self.position, dtype=np.float32)
        return (s * v) + p  # float32 multiply then add, as the loader does

    def triangles(self) -> np.ndarray:
        """(nt, 9) float32 world-space triangles."""
        if self.type == TRIANGLE:
            return np.asarray(self.vertices, dtype=np.float32).reshape(1, 9)
        w = self.world_vertices()
        return w[np.asarray(self.indices, dtype=np.int64)].reshape(-1, 9)

    def box(self) -> np.ndarray:
        w = self.world_vertices()
        return np.concatenate([w.min(axis=0), w.max(axis=0)]).astype(np.float32)


@dataclasses.dataclass
class SceneDesc:
    objects: list = dataclasses.field(default_factory=list)
    lights: list = dataclasses.field(default_factory=list)
    env: Optional[np.ndarray] = None  # (h, w, 3) float32
    volume: Optional[tuple] = None    # (sigma_s, sigma_a, g)
    name: str = "scene"
    camera: Optional[tuple] = None    # (position, yaw, pitch): the <camera> extension element
    texture: Optional[np.ndarray] = None  # (h, w, 3) float32 albedo texture (cupbr_scene_set_albedo_texture)
    terrain_chunks: int = 0               # heightfield scenes: the first objects are the terrain chunks
    terrain_extent: Optional[tuple] = None

    # -------------------------------------------------------------- build
    def add(self, obj: ObjectDesc) -> int:
        self.objects.append(obj)
        return len(self.objects) - 1

    def triangle_count(self) -> int:
        n = 0
        for o in self.objects:
            if o.type == MESH:
                n += len(o.indices)
            elif o.type == TRIANGLE:
                n += 1
        return n

    def build(self, bvh_params=None):
        """Commit to the GPU; returns a cupbr_b200.Scene."""
        from . import Scene
        return Scene.from_desc(self, bvh_params)

    def flat(self):
        """Yields (type, geo12, radius, material21, tris (nt,9) or None, box6 or None) per object."""
        for o in self.objects:
            geo = np.array([*o.p0, *o.p1, *o.p2, *o.p3], dtype=np.float32)
            tris = box = None
            if o.type in (MESH, TRIANGLE):
                tris = np.ascontiguousarray(o.triangles(), dtype=np.float32)
                if o.type == MESH:
                    box = o.box()
            yield o.type, geo, np.float32(o.radius), o.material.flat(), tris, box

    # ---------------------------------------------------------------- XML
    def to_xml(self, path: str, mesh_dir: Optional[str] = None) -> str:
        """Write cupbr scene XML (SceneLoader.cpp:140-454 schema) + OBJ meshes."""
        mesh_dir = mesh_dir or os.path.dirname(os.path.abspath(path))
        os.makedirs(mesh_dir, exist_ok=True)
        f = lambda v: ",".join(repr(float(np.float32(x))) for x in v)
        out = ["<header>", f"    <scene_size>{len(self.objects)}</scene_size>",
               f"    <light_count>{len(self.lights)}</light_count>", "</header>", "", "<geometry>"]
        for i, o in enumerate(self.objects):
            tag = f"geometry{i + 1}"
            out.append(f"    <{tag}>")
            out.append(f"        <type>{_GEO_NAMES[o.type]}</type>")
            if o.type == SPHERE:
                out += [f"        <position>{f(o.p0)}</position>", f"        <radius>{float(o.radius)!r}</radius>"]
            elif o.type == PLANE:
                out += [f"        <position>{f(o.p0)}</position>", f"        <normal>{f(o.p1)}</normal>"]
            elif o.type == QUAD:
                out += [f"        <position>{f(o.p0)}</position>", f"        <normal>{f(o.p1)}</normal>",
                        f"        <extend1>{f(o.p2)}</extend1>", f"        <extend2>{f(o.p3)}</extend2>"]
            elif o.type == TRIANGLE:
                v = np.asarray(o.vertices, dtype=np.float32).reshape(3, 3)
                out += [f"        <vertex{k + 1}>{f(v[k])}</vertex{k + 1}>" for k in range(3)]
            else:
                obj_name = f"{self.name}_{i + 1}.obj"
                obj_path = os.path.join(mesh_dir, obj_name)
                write_obj(obj_path, o.vertices, o.indices)
                out += [f"        <position>{f(o.position)}</position>", f"        <scale>{f(o.scale)}</scale>",
                        f"        <path>{obj_path}</path>"]
            m = o.material
            out += ["        <material>", f"            <type>{_MAT_NAMES[m.type]}</type>",
                    f"            <albedo_e>{f(m.albedo_e)}</albedo_e>", f"            <albedo_d>{f(m.albedo_d)}</albedo_d>",
                    f"            <albedo_s>{f(m.albedo_s)}</albedo_s>",
                    f"            <shininess>{float(m.shininess)!r}</shininess>",
                    f"            <roughness>{float(m.roughness)!r}</roughness>", f"            <eta>{float(m.eta)!r}</eta>",
                    f"            <sigma_s>{f(m.sigma_s)}</sigma_s>", f"            <sigma_a>{f(m.sigma_a)}</sigma_a>",
                    f"            <g>{float(m.g)!r}</g>"]
            if m.interface_glass:
                out.append("            <interface>GLASS</interface>")
            out += ["        </material>", f"    </{tag}>"]
        out += ["</geometry>", "", "<lights>"]
        for i, l in enumerate(self.lights):
            tag = f"light{i + 1}"
            out += [f"    <{tag}>", f"        <type>{'POINT' if l.type == POINT else 'AREA'}</type>",
                    f"        <position>{f(l.position)}</position>", f"        <intensity>{f(l.intensity)}</intensity>",
                    f"        <radiance>{f(l.radiance)}</radiance>", f"        <extend1>{f(l.half_extend1)}</extend1>",
                    f"        <extend2>{f(l.half_extend2)}</extend2>", f"    </{tag}>"]
        out.append("</lights>")
        if self.camera is not None:
            pos, yaw, pitch = self.camera
            out += ["", "<camera>", f"    <position>{f(pos)}</position>", f"    <yaw>{float(yaw)!r}</yaw>",
                    f"    <pitch>{float(pitch)!r}</pitch>", "</camera>"]
        if self.volume is not None:
            s, a, g = self.volume
            out += ["", "<volume>", f"    <sigma_s>{f(s)}</sigma_s>", f"    <sigma_a>{f(a)}</sigma_a>",
                    f"    <g>{float(g)!r}</g>", "</volume>"]
        if self.env is not None:
            env_path = os.path.join(mesh_dir, f"{self.name}_env.pfm")
            write_pfm(env_path, self.env)
            out += ["", "<environment>", f"    <path>{env_path}</path>", "</environment>"]
        with open(path, "w") as fh:
            fh.write("\n".join(out) + "\n")
        return path


def write_obj(path: str, vertices: np.ndarray, indices: np.ndarray) -> None:
    v = np.asarray(vertices, dtype=np.float32)
    idx = np.asarray(indices, dtype=np.int64) + 1
    with open(path, "w") as fh:
        fh.write("".join(f"v {a!r} {b!r} {c!r}\n" for a, b, c in v.astype(float).tolist()))
        fh.write("".join(f"f {a}/{a}/{a} {b}/{b}/{b} {c}/{c}/{c}\n" for a, b, c in idx.tolist()))


def write_pfm(path: str, rgb: np.ndarray) -> None:
    """Little-endian PFM; rgb[0] is the bottom row (the image's row 0)."""
    h, w, _ = rgb.shape
    with open(path, "wb") as fh:
        fh.write(f"PF\n{w} {h}\n-1.0\n".encode())
        fh.write(np.ascontiguousarray(rgb, dtype="<f4").tobytes())


def read_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as fh:
        assert fh.readline().strip() == b"PF"
        w, h = map(int, fh.readline().split())
        scale = float(fh.readline())
        data = np.frombuffer(fh.read(), dtype="<f4" if scale < 0 else ">f4")
    return data.reshape(h, w, 3).astype(np.float32)


# --------------------------------------------------------------- geometry

def cube() -> tuple[np.ndarray, np.ndarray]:
    """Unit cube [-1, 1]^3: 8 vertices, 12 outward-facing triangles."""
    v = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], dtype=np.float32)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    idx = []
    for a, b, c, d in quads:
        idx += [(a, b, c), (a, c, d)]
    idx = np.array(idx, dtype=np.uint32)
    # make every face point away from the centre
    for t in range(len(idx)):
        p = v[idx[t]]
        n = np.cross(p[1] - p[0], p[2] - p[0])
        if np.dot(n, p.mean(axis=0)) < 0:
            idx[t] = idx[t][[0, 2, 1]]
    return v, idx


def icosphere(subdiv: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4^subdiv outward-facing triangles."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in verts]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[k] = len(v) - 1
            return cache[k]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(v, dtype=np.float32)
    F = np.array(faces, dtype=np.uint32)
    n = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    flip = (n * V[F].mean(axis=1)).sum(axis=1) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    return V, F


def rotation_y(deg: float) -> np.ndarray:
    a = math.radians(deg)
    return np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]], dtype=np.float64)


# ---------------------------------------------------------------- scenes

def cornell_box(albedo_white=(0.73, 0.73, 0.73), red=(0.63, 0.065, 0.05), green=(0.14, 0.45, 0.09),
                light_radiance=(17.0, 12.0, 4.0)) -> SceneDesc:
    """Cornell box for the reference's default camera (origin, looking +z,
    90 degree vertical field of view): room x, y in [-1, 1], z in [1, 3]."""
    sc = SceneDesc(name="cornell")
    white = MaterialDesc(LAMBERT, albedo_d=tuple(albedo_white))
    sc.add(ObjectDesc(QUAD, white, p0=(0, -1, 2), p1=(0, 1, 0), p2=(1, 0, 0), p3=(0, 0, 1)))      # floor
    sc.add(ObjectDesc(QUAD, white, p0=(0, 1, 2), p1=(0, -1, 0), p2=(1, 0, 0), p3=(0, 0, 1)))      # ceiling
    sc.add(ObjectDesc(QUAD, MaterialDesc(LAMBERT, albedo_d=tuple(red)), p0=(-1, 0, 2), p1=(1, 0, 0),
                      p2=(0, 0, 1), p3=(0, 1, 0)))                                                 # left wall
    sc.add(ObjectDesc(QUAD, MaterialDesc(LAMBERT, albedo_d=tuple(green)), p0=(1, 0, 2), p1=(-1, 0, 0),
                      p2=(0, 1, 0), p3=(0, 0, 1)))                                                 # right wall
    sc.add(ObjectDesc(QUAD, white, p0=(0, 0, 3), p1=(0, 0, -1), p2=(1, 0, 0), p3=(0, 1, 0)))      # back wall
    v, idx = cube()
    for half, centre, deg in (((0.3, 0.3, 0.3), (0.35, -0.7, 1.8), -17.0),
                              ((0.3, 0.6, 0.3), (-0.33, -0.4, 2.35), 17.0)):
        w = (rotation_y(deg) @ (v.astype(np.float64) * np.array(half)).T).T + np.array(centre)
        sc.add(ObjectDesc(MESH, white, vertices=w.astype(np.float32), indices=idx.copy()))
    sc.lights.append(LightDesc(AREA, position=(0.0, 0.99, 2.0), radiance=tuple(light_radiance),
                               half_extend1=(0.125, 0.0, 0.0), half_extend2=(0.0, 0.0, 0.125)))
    return sc


def _hash01(ix: np.ndarray, iz: np.ndarray, seed: int) -> np.ndarray:
    """splitmix64-style integer hash of lattice points -> [0, 1) (wrapping uint64 arithmetic)."""
    with np.errstate(over="ignore"):
        x = (np.asarray(ix).astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)) ^ \
            (np.asarray(iz).astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F))
        x ^= np.uint64(seed) * np.uint64(0x165667B19E3779F9)
        x ^= x >> np.uint64(30)
        x *= np.uint64(0xBF58476D1CE4E5B9)
        x ^= x >> np.uint64(27)
        x *= np.uint64(0x94D049BB133111EB)
        x ^= x >> np.uint64(31)
    return (x >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def _value_noise(x: np.ndarray, z: np.ndarray, seed: int) -> np.ndarray:
    x0 = np.floor(x)
    z0 = np.floor(z)
    fx, fz = x - x0, z - z0
    sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
    ix, iz = x0.astype(np.int64) + (1 << 20), z0.astype(np.int64) + (1 << 20)
    a = _hash01(ix, iz, seed)
    b = _hash01(ix + 1, iz, seed)
    c = _hash01(ix, iz + 1, seed)
    d = _hash01(ix + 1, iz + 1, seed)
    return (a * (1 - sx) + b * sx) * (1 - sz) + (c * (1 - sx) + d * sx) * sz


def fbm(x: np.ndarray, z: np.ndarray, seed: int, octaves: int = 6, gain: float = 0.5, lacunarity: float = 2.0):
    r = np.zeros_like(x, dtype=np.float64)
    amp, freq = 1.0, 1.0
    for o in range(octaves):
        r += amp * (2.0 * _value_noise(x * freq, z * freq, seed * 131 + o) - 1.0)
        amp *= gain
        freq *= lacunarity
    return r


def terrain_height(x, z, seed: int = 0):
    return -1.5 + 1.2 * fbm(np.asarray(x, dtype=np.float64) / 6.0, np.asarray(z, dtype=np.float64) / 6.0, seed)


def sky_env(width: int = 2048, height: int = 1024, sun_dir=(0.35, 0.6, 0.72), sun_radiance=60.0) -> np.ndarray:
    """Procedural lat-long sky, rows indexed as direction2UV does
    (TracingDetail.h:185-196: row = (h-1) * acos(y)/pi, col = (w-1) * (atan2(z, x) + pi) / 2pi)."""
    theta = (np.arange(height, dtype=np.float64) + 0.5) / height * math.pi
    phi = (np.arange(width, dtype=np.float64) + 0.5) / width * 2 * math.pi - math.pi
    T, P = np.meshgrid(theta, phi, indexing="ij")
    dy = np.cos(T)
    dx = np.sin(T) * np.cos(P)
    dz = np.sin(T) * np.sin(P)
    up = np.clip(dy, 0.0, 1.0)[..., None]
    zenith = np.array([0.25, 0.45, 1.1])
    horizon = np.array([1.1, 1.05, 1.0])
    ground = np.array([0.12, 0.11, 0.10])
    sky = horizon * (1 - up) ** 3 + zenith * (1 - (1 - up) ** 3)
    img = np.where(dy[..., None] >= 0, sky, ground * (1 + 0.5 * np.clip(-dy, 0, 1))[..., None])
    s = np.asarray(sun_dir, dtype=np.float64)
    s /= np.linalg.norm(s)
    cosang = dx * s[0] + dy * s[1] + dz * s[2]
    sun = cosang > math.cos(math.radians(1.5))
    img[sun] = np.array([1.0, 0.95, 0.85]) * sun_radiance
    return img.astype(np.float32)


def random_material(rng: np.random.Generator) -> MaterialDesc:
    k = int(rng.integers(0, 3))
    if k == 0:
        return MaterialDesc(LAMBERT, albedo_d=tuple(rng.uniform(0.1, 0.9, 3).astype(np.float32).tolist()))
    if k == 1:
        return MaterialDesc(GGX, albedo_s=tuple(rng.uniform(0.5, 1.0, 3).astype(np.float32).tolist()),
                            roughness=float(np.float32(rng.uniform(0.05, 0.5))))
    return MaterialDesc(GLASS, albedo_s=(1.0, 1.0, 1.0), eta=1.5)


def heightfield_spheres(seed: int = 0, grid: int = 1024, crop: int = 1_000_000, n_spheres: int = 200,
                        subdiv: int = 4, chunk: int = 32, env_size=(2048, 1024), extent=(-20.0, 20.0, 1.0, 41.0),
                        ) -> SceneDesc:
    """The 1M-triangle benchmark scene (see module docstring)."""
    rng = np.random.default_rng(seed)
    sc = SceneDesc(name=f"hf{seed}")
    x0, x1, z0, z1 = extent
    xs = np.linspace(x0, x1, grid)
    zs = np.linspace(z0, z1, grid)
    Z, X = np.meshgrid(zs, xs, indexing="ij")
    Y = terrain_height(X, Z, seed)
    verts = np.stack([X, Y, Z], axis=-1).astype(np.float32)  # (row=z, col=x)
    nq = grid - 1
    tris_per_row = 2 * nq
    n_rows = min(nq, (crop + tris_per_row - 1) // tris_per_row)
    remaining = crop
    for r0 in range(0, n_rows, chunk):
        for c0 in range(0, nq, chunk):
            rows = range(r0, min(r0 + chunk, n_rows))
            cols = range(c0, min(c0 + chunk, nq))
            idx = []
            for r in rows:
                row_base = r * tris_per_row
                for c in cols:
                    for k in range(2):
                        t_global = row_base + 2 * c + k
                        if t_global >= crop:
                            continue
                        a, b = r * grid + c, r * grid + c + 1
                        d_, e = (r + 1) * grid + c, (r + 1) * grid + c + 1
                        # upward-facing winding (normal +y)
                        idx.append((a, d_, b) if k == 0 else (b, d_, e))
            if not idx:
                continue
            idx = np.array(idx, dtype=np.int64)
            used = np.unique(idx)
            remap = np.full(grid * grid, -1, dtype=np.int64)
            remap[used] = np.arange(len(used))
            v = verts.reshape(-1, 3)[used]
            sc.add(ObjectDesc(MESH, random_material(rng), vertices=v, indices=remap[idx].astype(np.uint32)))
            remaining -= len(idx)
    sc.terrain_chunks = len(sc.objects)
    sc.terrain_extent = (x0, x1, z0, z1)
    sv, sf = icosphere(subdiv)
    for _ in range(n_spheres):
        cx = rng.uniform(-9.0, 9.0)
        cz = rng.uniform(3.0, 18.0)
        rad = rng.uniform(0.2, 0.8)
        cy = float(terrain_height(cx, cz, seed)) + rad + rng.uniform(0.05, 0.6)
        sc.add(ObjectDesc(MESH, random_material(rng), vertices=sv.copy(), indices=sf.copy(),
                          position=(cx, cy, cz), scale=(rad, rad, rad)))
    sc.env = sky_env(*env_size)
    return sc


def material_test_scene(seed: int = 0, env_size=(64, 32)) -> SceneDesc:
    """Every geometry type (plane, quad, sphere, triangle, mesh), every
    material type (Lambert, Phong, mirror, glass, GGX, volume interface),
    a point and an area light and a small environment map, arranged in front
    of the default camera."""
    sc = SceneDesc(name=f"mixed{seed}")
    sc.add(ObjectDesc(PLANE, MaterialDesc(LAMBERT, albedo_d=(0.6, 0.6, 0.55)), p0=(0, -1, 0), p1=(0, 1, 0)))
    sc.add(ObjectDesc(QUAD, MaterialDesc(LAMBERT, albedo_d=(0.2, 0.5, 0.8)), p0=(0, 0.2, 4.5), p1=(0, 0, -1),
                      p2=(1.6, 0, 0), p3=(0, 1.1, 0)))
    mats = [MaterialDesc(LAMBERT, albedo_d=(0.8, 0.2, 0.2)),
            MaterialDesc(PHONG, albedo_d=(0.2, 0.2, 0.8), albedo_s=(1, 1, 1), shininess=51.2),
            MaterialDesc(MIRROR, albedo_s=(0.9, 0.9, 0.9)),
            MaterialDesc(GLASS, albedo_s=(1, 1, 1), eta=1.5),
            MaterialDesc(GGX, albedo_s=(1.0, 0.8, 0.9), roughness=0.1),
            MaterialDesc(GGX, albedo_s=(0.9, 0.9, 0.6), roughness=0.45)]
    for i, m in enumerate(mats):
        x = -1.5 + 0.6 * i
        sc.add(ObjectDesc(SPHERE, m, p0=(x, -0.72, 2.6 + 0.25 * (i % 2)), radius=0.27))
    sc.add(ObjectDesc(TRIANGLE, MaterialDesc(LAMBERT, albedo_d=(0.3, 0.8, 0.3), albedo_e=(0.4, 0.4, 0.1)),
                      vertices=np.array([[-1.2, 0.1, 3.2], [-0.4, 0.9, 3.4], [-0.2, 0.05, 3.0]], np.float32)))
    v, f = icosphere(1)
    sc.add(ObjectDesc(MESH, MaterialDesc(GGX, albedo_s=(0.95, 0.64, 0.54), roughness=0.2), vertices=v, indices=f,
                      position=(0.9, 0.35, 3.1), scale=(0.35, 0.35, 0.35)))
    vc, fc = cube()
    sc.add(ObjectDesc(MESH, MaterialDesc(VOLUME, interface_glass=1, eta=1.33), vertices=vc, indices=fc,
                      position=(0.1, 0.4, 2.2), scale=(0.2, 0.2, 0.2)))
    sc.lights.append(LightDesc(POINT, position=(0.5, 1.5, 1.5), intensity=(2.0, 2.0, 1.8)))
    sc.lights.append(LightDesc(AREA, position=(-0.5, 1.6, 2.5), radiance=(6.0, 5.0, 4.0),
                               half_extend1=(0.3, 0.0, 0.0), half_extend2=(0.0, 0.05, 0.2)))
    sc.env = sky_env(*env_size, sun_radiance=20.0)
    return sc


def volume_test_scene(scene_medium=((0.05, 0.04, 0.03), (0.02, 0.02, 0.02), 0.3)) -> SceneDesc:
    """Cornell box for the VOLUME method: a thin scene medium, one VOLUME
    sphere behind a glass interface (anisotropic HG), one VOLUME cube
    without interface, a mirror and a glass sphere, point + area light."""
    sc = cornell_box()
    sc.name = "volume"
    sc.objects = sc.objects[:5]  # the room
    sc.add(ObjectDesc(SPHERE, MaterialDesc(VOLUME, interface_glass=1, eta=1.33, sigma_s=(2.0, 1.5, 1.0),
                                           sigma_a=(0.1, 0.2, 0.3), g=0.5), p0=(-0.35, -0.6, 2.2), radius=0.35))
    vc, fc = cube()
    sc.add(ObjectDesc(MESH, MaterialDesc(VOLUME, sigma_s=(0.8, 0.8, 0.8), sigma_a=(0.3, 0.1, 0.1), g=-0.2),
                      vertices=vc, indices=fc, position=(0.45, -0.7, 1.8), scale=(0.25, 0.3, 0.25)))
    sc.add(ObjectDesc(SPHERE, MaterialDesc(MIRROR, albedo_s=(0.9, 0.9, 0.9)), p0=(0.5, 0.3, 2.5), radius=0.2))
    sc.add(ObjectDesc(SPHERE, MaterialDesc(GLASS, albedo_s=(1, 1, 1), eta=1.5), p0=(-0.1, 0.2, 1.6), radius=0.15))
    sc.lights.append(LightDesc(POINT, position=(0.0, 0.8, 1.5), intensity=(1.5, 1.5, 1.5)))
    sc.volume = scene_medium
    return sc


def perlin_grid(res: int = 256, seed: int = 0, octaves: int = 4, sigma_max: float = 8.0, scale: float = 4.0,
                ) -> np.ndarray:
    """Seeded 3-D gradient (Perlin) noise, `octaves` octaves (gain 0.5,
    lacunarity 2), mapped to densities in [0, sigma_max]: (res, res, res)
    float32 indexed [z, y, x] (x fastest in memory).

    Lattice point (x, y, z) of octave o gets the unit gradient
    g[perm[(perm[(perm[(x + 31 o) % 256] + y) % 256] + z) % 256]] (seeded
    permutation and gradients); voxel centres blend their cell's 8 corners
    with the quintic fade.  The gradients are tabulated per lattice point and
    the per-axis factors broadcast, so a 256^3 grid takes seconds."""
    rng = np.random.default_rng(seed)
    P = 256
    perm = rng.permutation(P)
    g = rng.normal(size=(P, 3))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    c = (np.arange(res, dtype=np.float64) + 0.5) / res
    total = np.zeros((res, res, res), dtype=np.float32)
    amp, freq, norm_ = 1.0, scale, 0.0
    fade = lambda t: t * t * t * (t * (t * 6 - 15) + 10)
    for o in range(octaves):
        f = c * freq
        i0 = np.floor(f).astype(np.int64)
        fr = f - i0
        w1 = fade(fr).astype(np.float32)
        w0 = (1.0 - fade(fr)).astype(np.float32)
        n = int(i0.max()) + 2  # lattice points per axis
        lat = np.arange(n)
        hx = perm[(lat + 31 * o) % P]
        hxy = perm[(hx[None, :] + lat[:, None]) % P]            # [y, x]
        hxyz = perm[(hxy[None, :, :] + lat[:, None, None]) % P]  # [z, y, x]
        gl = [np.ascontiguousarray(g[hxyz, k].astype(np.float32)).ravel() for k in range(3)]
        for dz in (0, 1):
            wz = (w1 if dz else w0)[:, None, None]
            fz = (fr - dz).astype(np.float32)[:, None, None]
            for dy in (0, 1):
                wy = (w1 if dy else w0)[None, :, None]
                fy = (fr - dy).astype(np.float32)[None, :, None]
                for dx in (0, 1):
                    wx = (w1 if dx else w0)[None, None, :]
                    fx = (fr - dx).astype(np.float32)[None, None, :]
                    idx = ((i0 + dz)[:, None, None] * n + (i0 + dy)[None, :, None]) * n + (i0 + dx)[None, None, :]
                    dot = gl[0].take(idx) * fx
                    dot += gl[1].take(idx) * fy
                    dot += gl[2].take(idx) * fz
                    dot *= (wz * wy) * wx * np.float32(amp)
                    total += dot
        norm_ += amp
        amp *= 0.5
        freq *= 2.0
    t = total / np.float32(norm_)
    lo, hi = float(t.min()), float(t.max())
    t = (t - np.float32(lo)) * np.float32(1.0 / max(hi - lo, 1e-12))
    return (np.float32(sigma_max) * t).astype(np.float32)


def cornell_variant(seed: int) -> SceneDesc:
    """A seeded variation of cornell_box(): wall colours, box sizes, positions
    and rotations, and light radiance drawn around the originals."""
    rng = np.random.default_rng(seed)
    jit = lambda c, a: tuple(float(np.clip(x + rng.uniform(-a, a), 0.02, 0.95)) for x in c)
    sc = cornell_box(albedo_white=jit((0.73, 0.73, 0.73), 0.1), red=jit((0.63, 0.065, 0.05), 0.1),
                     green=jit((0.14, 0.45, 0.09), 0.1),
                     light_radiance=tuple(float(v * rng.uniform(0.7, 1.3)) for v in (17.0, 12.0, 4.0)))
    v, idx = cube()
    boxes = [o for o in sc.objects if o.type == MESH]
    for o, (half, centre) in zip(boxes, (((0.3, 0.3, 0.3), (0.35, -0.7, 1.8)), ((0.3, 0.6, 0.3), (-0.33, -0.4, 2.35)))):
        h = np.array(half) * rng.uniform(0.8, 1.2)
        c = np.array(centre) + np.array([rng.uniform(-0.1, 0.1), 0.0, rng.uniform(-0.1, 0.1)])
        c[1] = -1.0 + h[1]
        w = (rotation_y(rng.uniform(-40.0, 40.0)) @ (v.astype(np.float64) * h).T).T + c
        o.vertices = w.astype(np.float32)
    sc.name = f"cornell_{seed}"
    return sc


def albedo_texture(size: int = 1024, seed=4) -> np.ndarray:
    """(size, size, 3) float32 albedo texture with texels U[0.2, 0.8]."""
    return np.random.default_rng(seed).uniform(0.2, 0.8, (size, size, 3)).astype(np.float32)


def with_texture(sc: SceneDesc, size: int = 1024, seed=4) -> SceneDesc:
    """Binds a seeded albedo texture (albedo_texture) to the scene's large
    surfaces by planar projection: a Cornell box's floor, ceiling and back
    wall (its white quads), a heightfield scene's terrain chunks (those with
    a Lambert material take the texel as their albedo)."""
    sc.texture = albedo_texture(size, seed)
    if sc.name.startswith("cornell"):
        frames = {0: ((-1.0, -1.0, 1.0), (2.0, 0.0, 0.0), (0.0, 0.0, 2.0)),   # floor
                  1: ((-1.0, 1.0, 1.0), (2.0, 0.0, 0.0), (0.0, 0.0, 2.0)),    # ceiling
                  4: ((-1.0, -1.0, 3.0), (2.0, 0.0, 0.0), (0.0, 2.0, 0.0))}   # back wall
        for i, f in frames.items():
            sc.objects[i].tex_frame = f
    elif sc.name.startswith("hf"):
        x0, x1, z0, z1 = sc.terrain_extent
        for o in sc.objects[:sc.terrain_chunks]:
            o.tex_frame = ((x0, 0.0, z0), (x1 - x0, 0.0, 0.0), (0.0, 0.0, z1 - z0))
    else:
        raise ValueError(f"no texture layout for scene {sc.name!r}")
    return sc


def medium_scene() -> SceneDesc:
    """The Cornell box of cornell_box() (walls, boxes, area light) as the
    surfaces around a heterogeneous medium filling the room interior."""
    sc = cornell_box()
    sc.name = "medium"
    return sc


def camera_for(width: int, height: int):
    """Camera(width, height) pose: Camera.cpp:6-11."""
    aspect = np.float32(width) / np.float32(height)
    return dict(position=(0.0, 0.0, 0.0), x_axis=(float(aspect), 0.0, 0.0), y_axis=(0.0, 1.0, 0.0),
                z_axis=(0.0, 0.0, 1.0), aspect_ratio=float(aspect))
