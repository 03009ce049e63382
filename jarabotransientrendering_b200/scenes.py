"""Seeded synthetic scenes for the transient path-tracing workloads.

The reference renders OBJ meshes given on its command line
(``src/bunnykiller.cpp:995-1002`` -> ``World::add_triangle_mesh``,
``src/RayTracing/World.h:209-541``).  It ships no benchmark scenes, so the
workloads are generated here from seeds and written out as plain OBJ files
that the reference's own loader accepts.

Conventions shared with the reference:

* geometric normal of a triangle (p0, p1, p2) is ``normalize(cross(p2-p0, p1-p0))``
  (``World.h:449``); every generator orients its triangles so that this normal
  points where the scene wants it (room walls inward, boxes and spheres outward);
* the rectangular area light is given by a corner point, a target point that
  defines its normal and a 2D size (``bunnykiller.cpp:1242-1262``) and builds its
  frame in ``RectangularAreaLightSource::setup`` (``RectangularAreaLightSource.h:66-80``);
* the pinhole camera basis is ``nv = normalize(focus - pos)``,
  ``uv = normalize(nv x up)``, ``vv = normalize(uv x nv)`` and the focal distance
  ``fd = 1 / tan(fov/2)`` (``PinholeCamera.h:56-75``, ``bunnykiller.cpp:1156-1161``).

Workloads (sizes from the benchmark configuration list):

* ``cornell``   - room of 10 triangles + two boxes of 12 triangles, point light,
  128x128, 1024 bins x 0.005, depth 6, 64 spp;
* ``icosphere`` - the same plus a displaced icosphere at subdivision 7
  (327,680 triangles), 512x512, 2048 bins x 0.0025, depth 8, 256 spp;
* ``medium``    - the Cornell scene in a homogeneous medium (sigma_a 0.05,
  sigma_s 0.5, HG g 0.3), 256x256, 4096 bins x 0.002, depth 12, 128 spp
  (8x8 strata x 2 paths per camera sample);
* ``guided``    - the Cornell scene with a GGX floor (alpha 0.2) and a
  0.05x0.05 area light hidden above an occluder slab, 512x512, 2048 bins.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional

import numpy as np

MAT_LAMBERTIAN = 0
MAT_GGX = 1

LIGHT_POINT = 0
LIGHT_RECT = 1

FLAG_ORTHONORMAL_FRAME = 1
FLAG_TIME_SAMPLING = 2       # "-time-sampling": time-based free flight, time-angular directions in media,
                             # total-time termination (the reference's SamplingMode::Transient)
FLAG_BIDIRECTIONAL = 4       # light subpaths + vertex connections (set_path_tracing_only(false)); needs
                             # FLAG_TIME_SAMPLING and no medium
COMP_DEPTH, COMP_POSITIONS, COMP_NORMALS = 2, 8, 16     # FilmComponents bits (FilmComponents.h)


@dataclasses.dataclass
class Material:
    kind: int
    kd: tuple
    alpha: float = 0.0


@dataclasses.dataclass
class Light:
    kind: int
    position: tuple          # point position, or rectangle corner
    intensity: tuple
    left: tuple = (0.0, 0.0, 0.0)
    up: tuple = (0.0, 0.0, 0.0)
    normal: tuple = (0.0, 0.0, 0.0)
    area: float = 0.0
    # CLI form of a rectangular light (kept so the reference can be driven)
    target: tuple = (0.0, 0.0, 0.0)
    size: tuple = (0.0, 0.0)


@dataclasses.dataclass
class Medium:
    sigma_a: tuple
    sigma_s: tuple
    g: float


@dataclasses.dataclass
class Camera:
    position: tuple
    focus: tuple
    up: tuple
    fov_deg: float
    focal_distance: Optional[float] = None   # overrides fov_deg when given

    def basis(self):
        """Float32 pinhole basis (nv, uv, vv, fd) as ``PinholeCamera.h:56-75`` builds it."""
        f32 = np.float32
        pos = np.array(self.position, f32)
        foc = np.array(self.focus, f32)
        up = np.array(self.up, f32)
        up = (up / np.sqrt(np.dot(up, up))).astype(f32)
        d = (foc - pos).astype(f32)
        nv = (d / np.sqrt(np.dot(d, d))).astype(f32)
        u = np.cross(nv, up).astype(f32)
        uv = (u / np.sqrt(np.dot(u, u))).astype(f32)
        v = np.cross(uv, nv).astype(f32)
        vv = (v / np.sqrt(np.dot(v, v))).astype(f32)
        if self.focal_distance is not None:
            fd = f32(self.focal_distance)
        else:
            fov = f32(math.pi / 180.0 * self.fov_deg / 2.0)
            fd = f32(1.0 / math.tan(float(fov)))
        return pos, nv, uv, vv, fd


@dataclasses.dataclass
class Mesh:
    name: str
    vertices: np.ndarray      # float32 [nv, 3]
    triangles: np.ndarray     # uint32 [nt, 3]
    material: int             # index into Scene.materials


@dataclasses.dataclass
class Scene:
    name: str
    meshes: List[Mesh]
    materials: List[Material]
    lights: List[Light]
    camera: Camera
    width: int
    height: int
    time_bins: int
    exposure: float
    offset: float
    max_bounces: int
    sqrt_spp: int
    incoming_samples: int
    medium: Optional[Medium] = None
    seed: int = 1
    flags: int = 0            # FLAG_ORTHONORMAL_FRAME: Lambertian sampling in an orthonormal frame
    camera_unwarp: int = 0    # bin by path time minus the camera-to-first-surface distance
    bounce_films: int = 0     # N > 0: per-bounce streak films (multibounce streak film)
    components: int = 0       # film components: COMP_DEPTH | COMP_POSITIONS | COMP_NORMALS

    # ---- flattened arrays (what the C ABI takes) -------------------------
    def flatten(self):
        verts, tris, mats = [], [], []
        base = 0
        for m in self.meshes:
            verts.append(np.asarray(m.vertices, np.float32))
            tris.append(np.asarray(m.triangles, np.uint32) + np.uint32(base))
            mats.append(np.full(len(m.triangles), m.material, np.uint32))
            base += len(m.vertices)
        return (np.ascontiguousarray(np.concatenate(verts)),
                np.ascontiguousarray(np.concatenate(tris)),
                np.ascontiguousarray(np.concatenate(mats)))

    @property
    def num_triangles(self):
        return int(sum(len(m.triangles) for m in self.meshes))

    @property
    def spp(self):
        return self.sqrt_spp * self.sqrt_spp

    def paths_per_frame(self):
        return self.width * self.height * self.spp * self.incoming_samples

    def write_obj(self, directory):
        """Write one OBJ per mesh (``v``/``f`` lines, 1-based indices) and return paths."""
        os.makedirs(directory, exist_ok=True)
        paths = []
        for m in self.meshes:
            p = os.path.join(directory, f"{self.name}_{m.name}.obj")
            with open(p, "w") as fh:
                fh.write(f"# {self.name}/{m.name}: {len(m.vertices)} vertices, {len(m.triangles)} triangles\n")
                for v in np.asarray(m.vertices, np.float32):
                    fh.write("v %.9g %.9g %.9g\n" % (v[0], v[1], v[2]))
                for t in np.asarray(m.triangles, np.int64):
                    fh.write("f %d %d %d\n" % (t[0] + 1, t[1] + 1, t[2] + 1))
            paths.append(p)
        return paths


# --------------------------------------------------------------------------
# geometry helpers
# --------------------------------------------------------------------------

def _ng(p0, p1, p2):
    """Reference geometric normal direction cross(p2-p0, p1-p0) (World.h:449)."""
    return np.cross(p2 - p0, p1 - p0)


def _orient(vertices, triangles, want):
    """Swap v1/v2 of every triangle whose reference normal points against ``want``.

    ``want`` is a per-triangle direction ([nt, 3]) the normal must agree with."""
    v = vertices.astype(np.float64)
    p0, p1, p2 = v[triangles[:, 0]], v[triangles[:, 1]], v[triangles[:, 2]]
    flip = np.einsum("ij,ij->i", _ng(p0, p1, p2), want) < 0
    out = triangles.copy()
    out[flip, 1], out[flip, 2] = triangles[flip, 2], triangles[flip, 1]
    return out


def _quad_tris(a, b, c, d):
    return [(a, b, c), (a, c, d)]


def room(size=1.0):
    """Open-front unit room: floor, ceiling, back, left, right (10 triangles).

    Returns a list of (name, vertices, triangles, inward normal)."""
    s = size
    faces = {
        "floor": ([(0, 0, 0), (s, 0, 0), (s, 0, s), (0, 0, s)], (0, 1, 0)),
        "ceiling": ([(0, s, 0), (s, s, 0), (s, s, s), (0, s, s)], (0, -1, 0)),
        "back": ([(0, 0, s), (s, 0, s), (s, s, s), (0, s, s)], (0, 0, -1)),
        "left": ([(0, 0, 0), (0, 0, s), (0, s, s), (0, s, 0)], (1, 0, 0)),
        "right": ([(s, 0, 0), (s, 0, s), (s, s, s), (s, s, 0)], (-1, 0, 0)),
    }
    out = []
    for name, (vs, n) in faces.items():
        v = np.array(vs, np.float32)
        t = np.array(_quad_tris(0, 1, 2, 3), np.uint32)
        t = _orient(v, t, np.tile(np.array(n, np.float64), (len(t), 1)))
        out.append((name, v, t))
    return out


def box(center_xz, size, angle_deg, y0=0.0):
    """Axis box of ``size`` (sx, sy, sz) resting on y0, rotated about +y, outward normals (12 triangles)."""
    sx, sy, sz = size
    hx, hz = sx / 2, sz / 2
    corners = np.array([[x, y, z] for y in (0.0, sy) for z in (-hz, hz) for x in (-hx, hx)], np.float64)
    a = math.radians(angle_deg)
    rot = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    pts = corners @ rot.T + np.array([center_xz[0], y0, center_xz[1]])
    # corner index = y*4 + z*2 + x
    quads = [(0, 1, 3, 2), (4, 5, 7, 6), (0, 1, 5, 4), (2, 3, 7, 6), (0, 2, 6, 4), (1, 3, 7, 5)]
    tris = []
    for q in quads:
        tris += _quad_tris(*q)
    t = np.array(tris, np.uint32)
    centre = pts.mean(axis=0)
    want = pts[t].mean(axis=1) - centre
    t = _orient(pts, t, want)
    return pts.astype(np.float32), t


def _icosahedron():
    p = (1 + 5 ** 0.5) / 2
    v = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p], [0, -1, -p],
                  [0, 1, -p], [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                  [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    return v / np.linalg.norm(v, axis=1, keepdims=True), f


def icosphere_unit(subdiv):
    """Unit icosphere: 20 * 4**subdiv faces, shared vertices (edge midpoints deduplicated)."""
    v, f = _icosahedron()
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m_idx = inv + len(v)
        nf = len(f)
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        ab, bc, ca = m_idx[:nf], m_idx[nf:2 * nf], m_idx[2 * nf:]
        v = np.concatenate([v, mid])
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1),
                            np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    return v, f


class ValueNoise3:
    """Seeded lattice value noise with smoothstep trilinear interpolation, values in [-1, 1]."""

    def __init__(self, seed):
        rng = np.random.default_rng(seed)
        self.perm = rng.permutation(256).astype(np.int64)
        self.vals = rng.uniform(-1.0, 1.0, 256)

    def _lattice(self, ix, iy, iz):
        p = self.perm
        return self.vals[p[(p[(p[ix & 255] + iy) & 255] + iz) & 255]]

    def __call__(self, x):
        i = np.floor(x).astype(np.int64)
        fr = x - i
        w = fr * fr * (3 - 2 * fr)
        out = 0.0
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    wt = ((w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1])
                          * (w[:, 2] if dz else 1 - w[:, 2]))
                    out = out + wt * self._lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
        return out


def displaced_icosphere(subdiv, centre, radius, amplitude=0.05, octaves=3, base_freq=2.0, seed=7):
    """Icosphere with radial value-noise displacement of ``amplitude`` * radius, outward normals."""
    v, f = icosphere_unit(subdiv)
    noise = ValueNoise3(seed)
    n = np.zeros(len(v))
    norm = 0.0
    for o in range(octaves):
        a = 0.5 ** o
        n += a * noise(v * base_freq * (2 ** o) + 17.0 * o)
        norm += a
    n /= norm
    r = radius * (1.0 + amplitude * n)
    pts = v * r[:, None] + np.asarray(centre, np.float64)
    t = f.astype(np.uint32)
    want = pts[t].mean(axis=1) - np.asarray(centre, np.float64)
    t = _orient(pts, t, want)
    return pts.astype(np.float32), t


def rect_light(corner, target, size, intensity):
    """Rectangular area light frame exactly as ``RectangularAreaLightSource::setup`` builds it."""
    f32 = np.float32
    p = np.array(corner, f32)
    d = (np.array(target, f32) - p).astype(f32)
    n = (d / np.sqrt(np.dot(d, d))).astype(f32)
    up = np.array([0, 1, 0], f32) if abs(float(np.dot(n, np.array([0, 1, 0], f32)))) < 0.9999 \
        else np.array([0, 0, 1], f32)
    left = np.cross(n, up).astype(f32)
    up = np.cross(n, left).astype(f32)
    left = (left * f32(size[0])).astype(f32)
    up = (up * f32(size[1])).astype(f32)
    area = float(f32(size[0]) * f32(size[1]))
    i = float(intensity)
    return Light(LIGHT_RECT, tuple(map(float, p)), (i, i, i), tuple(map(float, left)), tuple(map(float, up)),
                 tuple(map(float, n)), area, tuple(map(float, target)), tuple(map(float, size)))


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------

WHITE = (0.75, 0.75, 0.75)
RED = (0.75, 0.25, 0.25)
GREEN = (0.25, 0.75, 0.25)


def _cornell_meshes(seed, materials):
    """Cornell room (white/red/green walls) with a tall and a short box."""
    rng = np.random.default_rng(seed)
    jit = rng.uniform(-0.02, 0.02, 4) if seed != 1 else np.zeros(4)
    materials += [Material(MAT_LAMBERTIAN, WHITE), Material(MAT_LAMBERTIAN, RED),
                  Material(MAT_LAMBERTIAN, GREEN)]
    meshes = []
    for name, v, t in room():
        mat = {"left": 1, "right": 2}.get(name, 0)
        meshes.append(Mesh(name, v, t, mat))
    tv, tt = box((0.33 + jit[0], 0.62 + jit[1]), (0.3, 0.6, 0.3), 15.0)
    sv, st = box((0.66 + jit[2], 0.35 + jit[3]), (0.3, 0.3, 0.3), -18.0)
    meshes.append(Mesh("tallbox", tv, tt, 0))
    meshes.append(Mesh("shortbox", sv, st, 0))
    return meshes


def _default_camera():
    return Camera((0.5, 0.5, -1.37), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), 40.0)


def cornell(seed=1, width=128, height=128, time_bins=1024, exposure=0.005, max_bounces=6,
            sqrt_spp=8, incoming_samples=1):
    mats: List[Material] = []
    meshes = _cornell_meshes(seed, mats)
    light = Light(LIGHT_POINT, (0.5, 0.99, 0.5), (1.0, 1.0, 1.0))
    return Scene("cornell", meshes, mats, [light], _default_camera(), width, height, time_bins,
                 exposure, 0.0, max_bounces, sqrt_spp, incoming_samples, None, seed)


def icosphere(seed=1, subdiv=7, width=512, height=512, time_bins=2048, exposure=0.0025, max_bounces=8,
              sqrt_spp=16, incoming_samples=1, centre=(0.5, 0.32, 0.45)):
    mats: List[Material] = []
    meshes = _cornell_meshes(seed, mats)
    mats.append(Material(MAT_LAMBERTIAN, (0.6, 0.6, 0.6)))
    sv, st = displaced_icosphere(subdiv, centre, 0.25, 0.05, 3, 2.0, seed=1000 + seed)
    meshes.append(Mesh("icosphere", sv, st, len(mats) - 1))
    light = Light(LIGHT_POINT, (0.5, 0.99, 0.5), (1.0, 1.0, 1.0))
    return Scene("icosphere", meshes, mats, [light], _default_camera(), width, height, time_bins,
                 exposure, 0.0, max_bounces, sqrt_spp, incoming_samples, None, seed)


def medium(seed=1, width=256, height=256, time_bins=4096, exposure=0.002, max_bounces=12,
           sqrt_spp=8, incoming_samples=2, sigma_a=0.05, sigma_s=0.5, g=0.3):
    s = cornell(seed, width, height, time_bins, exposure, max_bounces, sqrt_spp, incoming_samples)
    s.name = "medium"
    s.medium = Medium((sigma_a,) * 3, (sigma_s,) * 3, g)
    return s


def guided(seed=1, width=512, height=512, time_bins=2048, exposure=0.0025, max_bounces=8,
           sqrt_spp=4, incoming_samples=1, floor_alpha=0.2, lambertian_floor=False):
    """GGX floor, small area light facing down, hidden above an occluder slab."""
    mats: List[Material] = []
    meshes = _cornell_meshes(seed, mats)
    if lambertian_floor:
        mats.append(Material(MAT_LAMBERTIAN, WHITE))
    else:
        mats.append(Material(MAT_GGX, (0.9, 0.9, 0.9), floor_alpha))
    meshes[0].material = len(mats) - 1          # floor
    rng = np.random.default_rng(5000 + seed)
    cx, cz = 0.5 + rng.uniform(-0.03, 0.03, 2)
    sv, st = box((cx, cz), (0.3, 0.02, 0.3), float(rng.uniform(-10, 10)), y0=0.93)
    meshes.append(Mesh("occluder", sv, st, 0))
    light = rect_light((0.525, 0.99, 0.525), (0.525, 0.0, 0.525), (0.05, 0.05), 40.0)
    return Scene("guided", meshes, mats, [light], _default_camera(), width, height, time_bins,
                 exposure, 0.0, max_bounces, sqrt_spp, incoming_samples, None, seed)


def batch_scene(index, seed=1):
    """One scene of the seeded 16-scene batch workload: a displaced icosphere (subdivision
    3..7, radius 0.2) in the Cornell room with its two boxes, every surface Lambertian with a
    seeded albedo in [0.2, 0.8]; point light below the ceiling; resolution 64^2..512^2, 256..4096
    time bins over the same 5.12 path-length units, 32..256 samples per pixel (non-square counts
    as sqrt_spp^2 x 2 incoming paths), depth 8; odd scenes fill the room with a homogeneous
    medium (sigma_s in [0.1, 1.0], sigma_a = sigma_s / 10, HG g in [-0.3, 0.6]).  Orthonormal
    Lambertian frames, so the learned proposal can be attached."""
    rng = np.random.default_rng(9000 + 131 * seed + index)
    subdiv = 3 + index % 5
    res = int(rng.choice((64, 128, 256, 512)))
    bins = int(rng.choice((256, 512, 1024, 2048, 4096)))
    # bound the film: at most 2^30 bins (6.4 GB FP64) per scene
    while res * res * bins > (1 << 30):
        bins //= 2
    sqrt_spp, inc = ((4, 2), (8, 1), (8, 2), (16, 1))[int(rng.integers(0, 4))]     # 32, 64, 128, 256 spp
    mats: List[Material] = []
    meshes = _cornell_meshes(seed + index, mats)
    for m in mats:
        a = rng.uniform(0.2, 0.8)
        m.kd = tuple(float(a * c / 0.75) for c in m.kd)
    mats.append(Material(MAT_LAMBERTIAN, (float(rng.uniform(0.2, 0.8)),) * 3))
    centre = (float(rng.uniform(0.35, 0.65)), 0.3, float(rng.uniform(0.3, 0.6)))
    sv, st = displaced_icosphere(subdiv, centre, 0.2, 0.05, 3, 2.0, seed=2000 + 17 * seed + index)
    meshes.append(Mesh("icosphere", sv, st, len(mats) - 1))
    light = Light(LIGHT_POINT, (0.5, 0.99, 0.5), (1.0, 1.0, 1.0))
    med = None
    if index % 2 == 1:
        sig_s = float(rng.uniform(0.1, 1.0))
        med = Medium((sig_s / 10,) * 3, (sig_s,) * 3, float(rng.uniform(-0.3, 0.6)))
    sc = Scene(f"batch{index:02d}", meshes, mats, [light], _default_camera(), res, res, bins, 5.12 / bins, 0.0, 8,
               sqrt_spp, inc, med, seed + index)
    sc.flags = FLAG_ORTHONORMAL_FRAME
    return sc


def batch_scenes(seed=1, n=16):
    """The seeded multi-scene workload (see ``batch_scene``)."""
    return [batch_scene(i, seed) for i in range(n)]


def small_batch_scenes(seed=1, n=64):
    """Many small scenes: the batch workload's scenes (see ``batch_scene``) at 64 x 64 pixels,
    256 time bins and 32 samples per pixel (4 x 4 camera samples x 2 incoming paths), i.e.
    131,072 paths each -- scenes too small to fill the GPU one at a time."""
    out = []
    for i in range(n):
        sc = batch_scene(i % 16, seed + i // 16)
        sc.width = sc.height = 64
        sc.time_bins = 256
        sc.exposure = 5.12 / 256
        sc.sqrt_spp, sc.incoming_samples = 4, 2
        sc.name = f"small{i:02d}"
        out.append(sc)
    return out


WORKLOADS = {"cornell": cornell, "icosphere": icosphere, "medium": medium, "guided": guided}


def random_rays(n, seed=0):
    """Correctness batch: origins U([0,1]^3), directions uniform on S^2, tnear 1e-5, tfar inf.

    Layout per ray: (ox, oy, oz, tnear, dx, dy, dz, tfar) float32."""
    rng = np.random.default_rng(seed)
    o = rng.random((n, 3))
    z = 1.0 - 2.0 * rng.random(n)
    phi = 2.0 * np.pi * rng.random(n)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = np.stack([s * np.cos(phi), s * np.sin(phi), z], 1)
    rays = np.empty((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e-5
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays
