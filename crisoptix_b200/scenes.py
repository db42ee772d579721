"""Procedural scenes for the Conditional ReSTIR PT frame loop.

The reference loads OBJ/FBX assets through assimp (src/Model.cpp:9-374); no
assets ship with it, so the workloads here are generated: the Cornell box
(small config) and a room of displaced icospheres with 256 emissive triangles
(large config).  Everything is seeded and deterministic.

A scene is a plain container of numpy arrays in the layout of
``crisb_scene_desc`` (include/crisb.h):

* positions / normals: float32 (V, 3)
* indices: uint32 (T, 3); triangle_material: uint32 (T,)
* materials: structured array with the ``crisb_material`` fields
* meshes (M, 2) = (first_triangle, num_triangles); instances: list of
  (mesh, material_override, 3x4 row-major transform)
* emitters: list of (color rgb, first_face, num_faces); emitter_faces (F, 9)

Material conventions follow the reference BRDF (shader/brdf.cu): with
spec_usage COLOR the specular F0 becomes the diffuse colour, so a
"Lambertian" material is the reference default roughness 1.0
(src/Model.cpp: roughness falls back to 1.0) and a "GGX" material has a
lower roughness.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, List, Tuple

import numpy as np

MATERIAL_DTYPE = np.dtype(
    [
        ("diffuse", "<f4", 3),
        ("specular", "<f4", 3),
        ("emission", "<f4", 3),
        ("roughness", "<f4"),
        ("spec_usage", "<i4"),
        ("reserved", "<i4"),
    ]
)


@dataclasses.dataclass
class Camera:
    """Camera(pos, viewDir, up, aspect, fov) of include/graph/Camera.h:24-79."""

    pos: Tuple[float, float, float]
    view_dir: Tuple[float, float, float]
    up: Tuple[float, float, float] = (0.0, 1.0, 0.0)
    aspect: float = 1.0
    fov: float = math.radians(60.0)
    changed: bool = False

    def rotate_around_origin(self, axis, angle: float) -> "Camera":
        """Camera::RotateAroundOrigin (src/Camera.cpp:34-38): rotate the
        position about `axis` through the origin and look at the origin."""
        a = np.asarray(axis, dtype=np.float64)
        a = a / np.linalg.norm(a)
        p = np.asarray(self.pos, dtype=np.float64)
        c, s = math.cos(angle), math.sin(angle)
        p2 = p * c + np.cross(a, p) * s + a * np.dot(a, p) * (1.0 - c)
        p2 = p2.astype(np.float32)
        d = -p2 / np.linalg.norm(p2)
        return Camera(tuple(float(v) for v in p2), tuple(float(v) for v in d), self.up, self.aspect, self.fov, True)


@dataclasses.dataclass
class Scene:
    positions: np.ndarray
    normals: np.ndarray
    indices: np.ndarray
    triangle_material: np.ndarray
    materials: np.ndarray
    meshes: np.ndarray
    instances: list
    emitters: list
    emitter_faces: np.ndarray
    name: str = "scene"
    # textured materials: (V, 2) vertex uvs, (H, W, 4) uint8 RGBA textures
    # (first row first) and (M, 3) int32 diffuse / specular / roughness
    # texture per material (-1: the material's constant)
    uvs: Optional[np.ndarray] = None
    textures: list = dataclasses.field(default_factory=list)
    material_textures: Optional[np.ndarray] = None

    @property
    def textured(self) -> bool:
        return self.material_textures is not None and bool((np.asarray(self.material_textures) >= 0).any())

    def flatten_uvs(self) -> np.ndarray:
        """(T, 6) corner uvs of the world-space triangles, in flatten() order."""
        UV = np.asarray(self.uvs, np.float32)[self.indices].reshape(-1, 6)
        if not self.instances:
            return UV.copy()
        return np.concatenate([UV[int(self.meshes[m][0]):int(self.meshes[m][0]) + int(self.meshes[m][1])]
                               for m, _, _ in self.instances]).astype(np.float32)

    @property
    def num_world_triangles(self) -> int:
        if not self.instances:
            return int(self.indices.shape[0])
        return int(sum(int(self.meshes[m][1]) for m, _, _ in self.instances))

    def flatten(self):
        """World-space triangle soup (T, 9) positions, (T, 9) normals, (T,)
        material; float64 math, for reference checks only."""
        P = self.positions[self.indices].reshape(-1, 9).astype(np.float64)
        N = self.normals[self.indices].reshape(-1, 9).astype(np.float64)
        if not self.instances:
            return P.astype(np.float32), N.astype(np.float32), self.triangle_material.copy()
        outp, outn, outm = [], [], []
        for mesh, override, xf in self.instances:
            first, count = (int(v) for v in self.meshes[mesh])
            M = np.asarray(xf, dtype=np.float64).reshape(3, 4)
            p = P[first:first + count].reshape(-1, 3) @ M[:, :3].T + M[:, 3]
            nt = np.linalg.inv(M[:, :3]).T
            n = N[first:first + count].reshape(-1, 3) @ nt.T
            n /= np.linalg.norm(n, axis=1, keepdims=True)
            outp.append(p.reshape(-1, 9))
            outn.append(n.reshape(-1, 9))
            mats = self.triangle_material[first:first + count]
            outm.append(np.full_like(mats, override) if override >= 0 else mats)
        return (np.concatenate(outp).astype(np.float32), np.concatenate(outn).astype(np.float32),
                np.concatenate(outm).astype(np.uint32))


def flat_scene(desc: Scene) -> Scene:
    """The same scene as a non-instanced triangle soup (float64 flattening)."""
    pos, nrm, mat = desc.flatten()
    T = len(mat)
    uvs = desc.flatten_uvs().reshape(-1, 2) if desc.uvs is not None else None
    return Scene(pos.reshape(-1, 3).copy(), nrm.reshape(-1, 3).copy(), np.arange(3 * T, dtype=np.uint32).reshape(T, 3),
                 mat.astype(np.uint32), desc.materials, np.zeros((0, 2), np.uint32), [], desc.emitters,
                 desc.emitter_faces, name=desc.name + "_flat", uvs=uvs, textures=desc.textures,
                 material_textures=desc.material_textures)


def _material(diffuse, roughness=1.0, emission=(0.0, 0.0, 0.0), specular=None):
    m = np.zeros((), dtype=MATERIAL_DTYPE)
    m["diffuse"] = diffuse
    m["specular"] = diffuse if specular is None else specular
    m["emission"] = emission
    m["roughness"] = roughness
    m["spec_usage"] = 0
    return m


class _Builder:
    def __init__(self):
        self.pos: List[np.ndarray] = []
        self.nrm: List[np.ndarray] = []
        self.mat: List[int] = []

    def tri(self, a, b, c, material: int, normal=None):
        a, b, c = (np.asarray(v, dtype=np.float32) for v in (a, b, c))
        if normal is None:
            n = np.cross(b - a, c - a)
            n = n / np.linalg.norm(n)
        else:
            n = np.asarray(normal, dtype=np.float32)
        self.pos.append(np.stack([a, b, c]))
        self.nrm.append(np.stack([n, n, n]).astype(np.float32))
        self.mat.append(material)

    def quad(self, a, b, c, d, material: int, normal):
        """Quad a-b-c-d as triangles (a,b,c) and (a,c,d), flat `normal`."""
        self.tri(a, b, c, material, normal)
        self.tri(a, c, d, material, normal)

    def box(self, lo, hi, material: int):
        x0, y0, z0 = lo
        x1, y1, z1 = hi
        self.quad((x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1), material, (0, 0, 1))
        self.quad((x1, y0, z0), (x0, y0, z0), (x0, y1, z0), (x1, y1, z0), material, (0, 0, -1))
        self.quad((x1, y0, z1), (x1, y0, z0), (x1, y1, z0), (x1, y1, z1), material, (1, 0, 0))
        self.quad((x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0), material, (-1, 0, 0))
        self.quad((x0, y1, z1), (x1, y1, z1), (x1, y1, z0), (x0, y1, z0), material, (0, 1, 0))
        self.quad((x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1), material, (0, -1, 0))

    def arrays(self):
        P = np.concatenate(self.pos).astype(np.float32)  # (3T, 3)
        N = np.concatenate(self.nrm).astype(np.float32)
        T = len(self.mat)
        idx = np.arange(3 * T, dtype=np.uint32).reshape(T, 3)
        return P, N, idx, np.asarray(self.mat, dtype=np.uint32)


def cornell_box() -> Tuple[Scene, Camera]:
    """Small config: unit-cube Cornell box, 5 wall quads (10 tris), a short
    Lambertian box and a tall GGX (roughness 0.3) box (12 tris each), and a
    0.25 x 0.25 ceiling light of radiance (17, 12, 4) (2 tris, one emitter)."""
    b = _Builder()
    mats = [
        _material((0.8, 0.8, 0.8)),  # 0 white
        _material((0.63, 0.065, 0.05)),  # 1 red
        _material((0.14, 0.45, 0.09)),  # 2 green
        _material((0.8, 0.8, 0.8)),  # 3 short box (Lambertian)
        _material((0.8, 0.8, 0.8), roughness=0.3),  # 4 tall box (GGX 0.3)
        _material((0.78, 0.78, 0.78), emission=(17.0, 12.0, 4.0)),  # 5 light
    ]
    x0, x1, y0, y1, z0, z1 = -0.5, 0.5, 0.0, 1.0, -0.5, 0.5
    b.quad((x0, y0, z1), (x1, y0, z1), (x1, y0, z0), (x0, y0, z0), 0, (0, 1, 0))  # floor
    b.quad((x0, y1, z0), (x1, y1, z0), (x1, y1, z1), (x0, y1, z1), 0, (0, -1, 0))  # ceiling
    b.quad((x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0), 0, (0, 0, 1))  # back
    b.quad((x0, y0, z1), (x0, y0, z0), (x0, y1, z0), (x0, y1, z1), 1, (1, 0, 0))  # left, red
    b.quad((x1, y0, z0), (x1, y0, z1), (x1, y1, z1), (x1, y1, z0), 2, (-1, 0, 0))  # right, green
    b.box((0.04, 0.0, -0.06), (0.34, 0.3, 0.24), 3)
    b.box((-0.36, 0.0, -0.38), (-0.06, 0.6, -0.08), 4)
    ly = 0.999
    h = 0.125
    light_first = len(b.mat)
    b.quad((-h, ly, -h), (h, ly, -h), (h, ly, h), (-h, ly, h), 5, (0, -1, 0))
    P, N, idx, tm = b.arrays()
    faces = P[3 * light_first:3 * light_first + 6].reshape(2, 9)
    scene = Scene(P, N, idx, tm, np.stack(mats), np.zeros((0, 2), np.uint32), [],
                  [((17.0, 12.0, 4.0), 0, 2)], faces.astype(np.float32), name="cornell")
    cam = Camera((0.0, 0.5, 1.35), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 1.0, math.radians(60.0))
    return scene, cam


def _checker(h: int, w: int, a, b, cell: int = 1) -> np.ndarray:
    yy, xx = np.mgrid[0:h, 0:w]
    on = ((yy // cell + xx // cell) % 2 == 0)[..., None]
    return np.where(on, np.asarray(a, np.uint8), np.asarray(b, np.uint8)).astype(np.uint8)


def textured_cornell_box() -> Tuple[Scene, Camera]:
    """The Cornell box with textured materials: a checkered diffuse floor and
    back wall (8 x 8 texels, uvs running over [-1.5, 1.5] so the wrap is
    exercised), a 5 x 3 diffuse gradient on the short box, an
    occlusion-roughness-metal texture (g = roughness, b = metal, 4 x 4) on the
    tall box's specular input with SpecTexUsage::OccRoughMetal, and a 6 x 6
    roughness texture on the red wall, which gets a specular colour.  uvs are
    planar projections of the vertex positions."""
    desc, cam = cornell_box()
    mats = desc.materials.copy()
    mats[1]["specular"] = (0.9, 0.9, 0.9)
    mats[4]["spec_usage"] = 1  # CRISB_SPEC_OCC_ROUGH_METAL
    P, N = desc.positions, desc.normals
    ax = np.argmax(np.abs(N), axis=1)
    u = np.where(ax == 0, P[:, 2], P[:, 0])
    v = np.where(ax == 1, P[:, 2], P[:, 1])
    uvs = (np.stack([u, v], axis=1) * 3.0).astype(np.float32)
    rng = np.random.default_rng(3)
    gradient = np.zeros((3, 5, 4), np.uint8)
    gradient[..., 0] = np.linspace(40, 250, 5, dtype=np.uint8)[None, :]
    gradient[..., 1] = np.linspace(200, 30, 3, dtype=np.uint8)[:, None]
    gradient[..., 2] = 90
    gradient[..., 3] = 255
    orm = np.zeros((4, 4, 4), np.uint8)
    orm[..., 0] = 255
    orm[..., 1] = rng.integers(50, 230, (4, 4))
    orm[..., 2] = rng.integers(0, 256, (4, 4))
    orm[..., 3] = 255
    rough = np.zeros((6, 6, 4), np.uint8)
    rough[..., 0] = rng.integers(40, 255, (6, 6))
    rough[..., 3] = 255
    textures = [_checker(8, 8, (230, 230, 220, 255), (40, 60, 160, 255), 2), gradient, orm, rough]
    mt = np.full((len(mats), 3), -1, np.int32)
    mt[0, 0] = 0  # floor, ceiling and back wall: checker diffuse
    mt[3, 0] = 1  # short box: gradient diffuse
    mt[4, 1] = 2  # tall box: ORM specular input
    mt[1, 2] = 3  # red wall: roughness texture
    return dataclasses.replace(desc, materials=mats, uvs=uvs, textures=textures, material_textures=mt,
                               name="cornell_textured"), cam


def _icosphere(subdiv: int):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], dtype=np.float64)
    f = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
                  (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
                  (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (len(v) + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // (len(v) + 1), uniq % (len(v) + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01, m12, m20 = (inv[:nf] + base), (inv[nf:2 * nf] + base), (inv[2 * nf:] + base)
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f


def _hash3(ix, iy, iz, seed):
    h = (ix.astype(np.uint32) * np.uint32(0x8DA6B343)) ^ (iy.astype(np.uint32) * np.uint32(0xD8163841)) ^ \
        (iz.astype(np.uint32) * np.uint32(0xCB1AB31F)) ^ np.uint32(seed * 0x9E3779B9 & 0xFFFFFFFF)
    h ^= h >> np.uint32(16)
    h *= np.uint32(0x7FEB352D)
    h ^= h >> np.uint32(15)
    h *= np.uint32(0x846CA68B)
    h ^= h >> np.uint32(16)
    return h.astype(np.float64) / 4294967295.0 * 2.0 - 1.0


def _value_noise(p, seed):
    pf = np.floor(p)
    i = pf.astype(np.int64)
    w = p - pf
    w = w * w * (3.0 - 2.0 * w)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                c = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                wx = w[:, 0] if dx else 1.0 - w[:, 0]
                wy = w[:, 1] if dy else 1.0 - w[:, 1]
                wz = w[:, 2] if dz else 1.0 - w[:, 2]
                out += c * wx * wy * wz
    return out


def _fbm(p, seed, octaves=4):
    total, amp, freq, norm = np.zeros(len(p)), 1.0, 1.0, 0.0
    for o in range(octaves):
        total += amp * _value_noise(p * freq, seed + 17 * o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def displaced_icosphere(subdiv: int, amplitude: float, seed: int, frequency: float = 2.0):
    """Unit icosphere with `subdiv` subdivisions (20 * 4**subdiv faces),
    vertices displaced along the normal by amplitude * fBm (4 octaves of value
    noise); smooth area-weighted vertex normals."""
    v, f = _icosphere(subdiv)
    v = v * (1.0 + amplitude * _fbm(v * frequency, seed))[:, None]
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    vn = np.zeros_like(v)
    for c in range(3):
        np.add.at(vn, f[:, c], fn)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    return v.astype(np.float32), vn.astype(np.float32), f.astype(np.uint32)


def sphere_room(num_spheres: int = 64, subdiv: int = 5, num_emitters: int = 256, seed: int = 1,
                room=(20.0, 8.0, 20.0), aspect: float = 16.0 / 9.0) -> Tuple[Scene, Camera]:
    """Large config: a room of `room` size centred on the origin, `num_spheres`
    instances of one displaced icosphere (radius U[0.2, 1.0], fBm amplitude
    0.1 * radius), `num_emitters` emissive triangles under the ceiling with
    radiance U[1, 20] per channel (one emitter each), half the spheres
    Lambertian (albedo U[0.1, 0.9]^3, roughness 1), half GGX (roughness
    U[0.05, 0.8])."""
    rng = np.random.default_rng(seed)
    hx, hy, hz = room[0] / 2, room[1] / 2, room[2] / 2
    sv, sn, sf = displaced_icosphere(subdiv, 0.1, seed)
    b = _Builder()
    mats = [_material((0.7, 0.7, 0.7))]  # 0: room
    b.quad((-hx, -hy, hz), (hx, -hy, hz), (hx, -hy, -hz), (-hx, -hy, -hz), 0, (0, 1, 0))
    b.quad((-hx, hy, -hz), (hx, hy, -hz), (hx, hy, hz), (-hx, hy, hz), 0, (0, -1, 0))
    b.quad((-hx, -hy, -hz), (hx, -hy, -hz), (hx, hy, -hz), (-hx, hy, -hz), 0, (0, 0, 1))
    b.quad((hx, -hy, hz), (-hx, -hy, hz), (-hx, hy, hz), (hx, hy, hz), 0, (0, 0, -1))
    b.quad((-hx, -hy, hz), (-hx, -hy, -hz), (-hx, hy, -hz), (-hx, hy, hz), 0, (1, 0, 0))
    b.quad((hx, -hy, -hz), (hx, -hy, hz), (hx, hy, hz), (hx, hy, -hz), 0, (-1, 0, 0))
    sphere_mats = []
    for i in range(num_spheres):
        albedo = rng.uniform(0.1, 0.9, 3)
        if i % 2 == 0:
            sphere_mats.append(_material(albedo, roughness=1.0))
        else:
            sphere_mats.append(_material(albedo, roughness=float(rng.uniform(0.05, 0.8))))
    mats.extend(sphere_mats)
    emit_first = len(b.mat)
    emitters = []
    ey = hy - 0.05
    for e in range(num_emitters):
        radiance = rng.uniform(1.0, 20.0, 3)
        cx, cz = rng.uniform(-hx + 0.5, hx - 0.5), rng.uniform(-hz + 0.5, hz - 0.5)
        ang = rng.uniform(0, 2 * math.pi)
        s = 0.25
        pts = [(cx + s * math.cos(ang + k * 2 * math.pi / 3), ey, cz + s * math.sin(ang + k * 2 * math.pi / 3))
               for k in range(3)]
        mats.append(_material((0.5, 0.5, 0.5), emission=tuple(radiance)))
        # wind so the face normal points down (-y)
        a, bb, c = (np.asarray(p, np.float32) for p in pts)
        if np.cross(bb - a, c - a)[1] > 0:
            bb, c = c, bb
        b.tri(a, bb, c, len(mats) - 1, (0, -1, 0))
        emitters.append((tuple(float(x) for x in radiance), e, 1))
    P, N, idx, tm = b.arrays()
    faces = P[3 * emit_first:].reshape(-1, 9).astype(np.float32)
    n_room_tris = len(tm)
    # sphere mesh appended after the room/emitter triangles
    base_v = len(P)
    P = np.concatenate([P, sv])
    N = np.concatenate([N, sn])
    idx = np.concatenate([idx, sf + base_v])
    tm = np.concatenate([tm, np.full(len(sf), 1, np.uint32)])
    meshes = np.array([(0, n_room_tris), (n_room_tris, len(sf))], dtype=np.uint32)
    instances = [(0, -1, [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0])]
    for i in range(num_spheres):
        r = float(rng.uniform(0.2, 1.0))
        c = (float(rng.uniform(-hx + r, hx - r)), float(rng.uniform(-hy + r, hy - r)),
             float(rng.uniform(-hz + r, hz - r)))
        instances.append((1, 1 + i, [r, 0, 0, c[0], 0, r, 0, c[1], 0, 0, r, c[2]]))
    scene = Scene(P.astype(np.float32), N.astype(np.float32), idx.astype(np.uint32), tm, np.stack(mats), meshes,
                  instances, emitters, faces, name=f"sphere_room_{num_spheres}x{20 * 4 ** subdiv}")
    # inside the room, 80% of the way to the +z wall, looking at the origin
    pos = np.array([0.0, 0.125 * hy, 0.8 * hz], np.float32)
    d = -pos / np.linalg.norm(pos)
    cam = Camera(tuple(float(v) for v in pos), tuple(float(v) for v in d), (0.0, 1.0, 0.0), aspect,
                 math.radians(60.0))
    return scene, cam


def orbit_camera(cam: Camera, frame: int, frames_per_orbit: int = 60) -> Camera:
    """Frame `frame` of a camera orbit about the y axis through the origin
    (Camera::RotateAroundOrigin applied once per frame)."""
    if frame == 0:
        return cam
    c = cam
    for _ in range(frame):
        c = c.rotate_around_origin((0.0, 1.0, 0.0), 2.0 * math.pi / frames_per_orbit)
    return c


# Multiview config: 8 views at 512x512, 4 at 1280x720, 4 at 1920x1080.
MULTIVIEW_RESOLUTIONS = [(512, 512)] * 8 + [(1280, 720)] * 4 + [(1920, 1080)] * 4


def multiview_cameras(resolutions=None, radius: float = 12.0, room=(20.0, 8.0, 20.0), seed: int = 2,
                      fov: float = math.radians(60.0)):
    """One camera per resolution on a sphere of `radius` about the room centre,
    seeded jittered directions, each looking at the centre.  Positions are
    scaled into the room's interior (80% of each half extent) when the sphere
    reaches outside it, so every camera sees the scene from inside."""
    res = list(resolutions or MULTIVIEW_RESOLUTIONS)
    rng = np.random.default_rng(seed)
    n = len(res)
    out = []
    for k, (w, h) in enumerate(res):
        # stratified directions (golden-angle spiral) with a seeded jitter
        z = 1.0 - 2.0 * (k + 0.5) / n + rng.uniform(-0.5, 0.5) / n
        phi = k * math.pi * (3.0 - math.sqrt(5.0)) + rng.uniform(-0.2, 0.2)
        r = math.sqrt(max(0.0, 1.0 - z * z))
        d = np.array([r * math.cos(phi), 0.7 * z, r * math.sin(phi)])
        d /= np.linalg.norm(d)
        pos = d * radius
        lim = 0.8 * np.array(room) / 2.0
        scale = min(1.0, float(np.min(lim / np.maximum(np.abs(pos), 1e-9))))
        pos = pos * scale
        view = -pos / np.linalg.norm(pos)
        out.append((Camera(pos=tuple(float(v) for v in pos), view_dir=tuple(float(v) for v in view),
                           up=(0.0, 1.0, 0.0), aspect=w / h, fov=fov, changed=False), w, h))
    return out
