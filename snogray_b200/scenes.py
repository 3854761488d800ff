"""Scene data and the seeded synthetic workloads the renderer is measured on.

A `SceneData` holds a scene as flat numpy arrays, in the shape the C ABI's
`SnogSceneDesc` takes them (include/snogray_b200.h).  Primitive ids follow the
reference's order of insertion into the acceleration structure
(surface/surface-group.cc:66-71, surface/mesh.cc:1093-1108): mesh triangles by
part, then spheres, then tripars.

Material records mirror the reference constructors:
  Lambert(color)                               material/lambert.h
  CookTorrance(color, gloss_color, m, ior)     material/cook-torrance.h:27-30
  Mirror(ior, reflectance, color)              material/mirror.h:47-49
  Glass(Medium(ior, absorb))                   material/glass.h:27, medium.h:30
  Glow(color[, underlying])                    material/glow.h:28-30
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MAT_LAMBERT, MAT_COOK_TORRANCE, MAT_MIRROR, MAT_GLASS, MAT_GLOW = range(5)

# One material record: type, color[3], gloss[3], m, ior_n, ior_k, absorb[3],
# underlying.  Stored as a structured array so it can be handed to C as-is.
MAT_DTYPE = np.dtype([("type", "<u4"), ("color", "<f4", 3), ("gloss", "<f4", 3),
                      ("m", "<f4"), ("ior_n", "<f4"), ("ior_k", "<f4"),
                      ("absorb", "<f4", 3), ("underlying", "<i4")])
SPHERE_DTYPE = np.dtype([("center", "<f4", 3), ("radius", "<f4"), ("mat", "<u4")])
TRIPAR_DTYPE = np.dtype([("v0", "<f4", 3), ("e1", "<f4", 3), ("e2", "<f4", 3),
                         ("parallelogram", "<u4"), ("mat", "<u4")])
PLIGHT_DTYPE = np.dtype([("pos", "<f4", 3), ("color", "<f4", 3), ("angle", "<f4"),
                         ("fringe_angle", "<f4"), ("dir", "<f4", 3)])
FLIGHT_DTYPE = np.dtype([("dir", "<f4", 3), ("angle", "<f4"), ("color", "<f4", 3)])


def _f32(x):
    return np.float32(x)


@dataclass
class Camera:
    """Pinhole camera in the reference's representation (camera/camera.h).

    `point()` and `set_vert_fov()` follow Camera::_point (camera.h:114-128) and
    Camera::set_fov (camera.h:231-242) for a film format of the image's aspect
    ratio, in float32 like the reference's dist_t.
    """
    pos: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    forward: np.ndarray = field(default_factory=lambda: np.array([0, 0, 1], np.float32))
    right: np.ndarray = field(default_factory=lambda: np.array([1, 0, 0], np.float32))
    up: np.ndarray = field(default_factory=lambda: np.array([0, 1, 0], np.float32))
    tan_half_fov_x: float = 0.0
    tan_half_fov_y: float = 0.0

    @staticmethod
    def _unit(v):
        v = np.asarray(v, np.float32)
        return (v * _f32(1.0 / np.float32(np.sqrt(np.float32(np.dot(v, v)))))).astype(np.float32)

    def move(self, pos):
        self.pos = np.asarray(pos, np.float32)

    def point(self, target, user_up):
        d = self._unit(np.asarray(target, np.float32) - self.pos)
        user_up = np.asarray(user_up, np.float32)
        self.forward = d
        self.right = self._unit(np.cross(user_up, d))
        self.up = self._unit(np.cross(d, self.right))

    def set_vert_fov(self, fov, aspect):
        t = math.tan(fov / 2)
        self.tan_half_fov_y = float(_f32(t))
        self.tan_half_fov_x = float(_f32(t * aspect))


@dataclass
class SceneData:
    materials: np.ndarray
    vertices: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    triangles: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.uint32))
    tri_mat: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    spheres: np.ndarray = field(default_factory=lambda: np.zeros(0, SPHERE_DTYPE))
    tripars: np.ndarray = field(default_factory=lambda: np.zeros(0, TRIPAR_DTYPE))
    point_lights: np.ndarray = field(default_factory=lambda: np.zeros(0, PLIGHT_DTYPE))
    far_lights: np.ndarray = field(default_factory=lambda: np.zeros(0, FLIGHT_DTYPE))
    envmap: np.ndarray | None = None          # (H, W, 3) float32, row 0 = top
    env_frame: np.ndarray = field(default_factory=lambda: np.eye(3, dtype=np.float32))
    name: str = "scene"
    normals: np.ndarray | None = None          # (n_vertices, 3) float32 vertex normals
    right_handed: bool = False                 # mesh normal e1 x e2 (PLY meshes)

    def __post_init__(self):
        self.vertices = np.ascontiguousarray(self.vertices, np.float32).reshape(-1, 3)
        self.triangles = np.ascontiguousarray(self.triangles, np.uint32).reshape(-1, 3)
        self.tri_mat = np.ascontiguousarray(self.tri_mat, np.uint32).reshape(-1)
        if self.tri_mat.size and np.any(np.diff(self.tri_mat.astype(np.int64)) < 0):
            raise ValueError("tri_mat must be non-decreasing (one mesh part per material run)")
        if self.envmap is not None:
            self.envmap = np.ascontiguousarray(self.envmap, np.float32)
        if self.normals is not None:
            self.normals = np.ascontiguousarray(self.normals, np.float32).reshape(-1, 3)

    @property
    def n_prims(self):
        return len(self.triangles) + len(self.spheres) + len(self.tripars)


@dataclass
class RenderParams:
    """ValTable keys of the reference's path integrator and image output
    (render/path-integ.cc:64-68, render-params.h:32-36,
    global-render-state.cc:37-38)."""
    width: int = 256
    height: int = 256
    spp: int = 16                      # samples
    min_path_len: int = 3              # surface_integ.min_path_len
    max_path_len: int = 25             # surface_integ.max_path_len
    direct_samples: int = 1            # surface_integ.direct_samples
    min_trace: float = 1e-3            # min_trace
    bg_alpha: float = 1.0              # background_alpha
    seed: int = 0
    integrator: int = 0                # surface_integ.type: 0 path, 1 direct (direct_samples =
                                       # surface_integ.light_samples)
    flags: int = 0                     # SNOG_RENDER_* bits (1: count traversal nodes and tests)


def material(mtype, color=(0, 0, 0), gloss=(1, 1, 1), m=0.0, ior_n=1.5, ior_k=0.0,
             absorb=(0, 0, 0), underlying=-1):
    r = np.zeros((), MAT_DTYPE)
    r["type"], r["color"], r["gloss"], r["m"] = mtype, color, gloss, m
    r["ior_n"], r["ior_k"], r["absorb"], r["underlying"] = ior_n, ior_k, absorb, underlying
    return r


def _mats(recs):
    return np.array([r[()] for r in recs], MAT_DTYPE)


# ---------------------------------------------------------------------------
# Cornell-style box: 5 axis-aligned quads (10 triangles, 3 Lambert parts), a
# Lambert sphere and a Glass sphere of radius 0.3, and a 0.25 x 0.25
# parallelogram area light of radiance 15 just below the ceiling.

def cornell_box():
    mats = _mats([
        material(MAT_LAMBERT, (0.73, 0.73, 0.73)),   # 0 white
        material(MAT_LAMBERT, (0.65, 0.05, 0.05)),   # 1 red
        material(MAT_LAMBERT, (0.12, 0.45, 0.15)),   # 2 green
        material(MAT_GLASS, ior_n=1.5),              # 3 glass, Medium(1.5)
        material(MAT_GLOW, (15.0, 15.0, 15.0)),      # 4 light
    ])
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1],      # floor y=0
                  [0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1]],     # ceiling y=1
                 np.float32)
    tris = np.array([
        [0, 1, 2], [0, 2, 3],      # floor
        [4, 6, 5], [4, 7, 6],      # ceiling
        [3, 2, 6], [3, 6, 7],      # back wall z=1
        [0, 3, 7], [0, 7, 4],      # left wall x=0 (red)
        [1, 5, 6], [1, 6, 2],      # right wall x=1 (green)
    ], np.uint32)
    tri_mat = np.array([0, 0, 0, 0, 0, 0, 1, 1, 2, 2], np.uint32)
    spheres = np.zeros(2, SPHERE_DTYPE)
    spheres[0] = ((0.3, 0.3, 0.65), 0.3, 0)
    spheres[1] = ((0.7, 0.6, 0.3), 0.3, 3)
    tripars = np.zeros(1, TRIPAR_DTYPE)
    # normal = e2 x e1 (surface/tripar.cc:54) points down, into the room.
    tripars[0] = ((0.375, 0.999, 0.375), (0, 0, 0.25), (0.25, 0, 0), 1, 4)
    return SceneData(materials=mats, vertices=v, triangles=tris, tri_mat=tri_mat,
                     spheres=spheres, tripars=tripars, name="cornell")


def cornell_camera(width, height):
    cam = Camera()
    cam.move((0.5, 0.5, -1.2))
    cam.point((0.5, 0.5, 0.5), (0, 1, 0))
    cam.set_vert_fov(math.radians(40.0), width / height)
    return cam


def cornell_params(width=256, height=256, spp=16, seed=0):
    return RenderParams(width=width, height=height, spp=spp, min_path_len=3, max_path_len=8,
                        direct_samples=1, seed=seed)


def direct_params(width=128, height=128, spp=16, seed=0, light_samples=4):
    """The direct-lighting integrator (surface_integ.type = direct) with
    LIGHT_SAMPLES samples per light."""
    return RenderParams(width=width, height=height, spp=spp, direct_samples=light_samples, integrator=1,
                        seed=seed)


# ---------------------------------------------------------------------------
# The Cornell walls with the remaining materials and lights of the path:
# Mirror surfaces (the conductor Ior(0.25, 3) that material.mirror uses by
# default, material/material.lua:232; a dielectric one over a Lambert; one of
# zero reflectance, which always samples its underlying Lambert,
# material/mirror.cc:70-80), a glowing sphere (SphereLightSampler,
# light/sphere-light-sampler.cc:40-194) and an omni point light
# (light/point-light.cc:78-107).

def _cornell_walls():
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1],
                  [0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1]], np.float32)
    tris = np.array([[0, 1, 2], [0, 2, 3], [4, 6, 5], [4, 7, 6], [3, 2, 6], [3, 6, 7],
                     [0, 3, 7], [0, 7, 4], [1, 5, 6], [1, 6, 2]], np.uint32)
    tri_mat = np.array([0, 0, 0, 0, 0, 0, 1, 1, 2, 2], np.uint32)
    return v, tris, tri_mat


def mirror_scene():
    mats = _mats([
        material(MAT_LAMBERT, (0.73, 0.73, 0.73)),                              # 0 white
        material(MAT_LAMBERT, (0.65, 0.05, 0.05)),                              # 1 red
        material(MAT_LAMBERT, (0.12, 0.45, 0.15)),                              # 2 green
        material(MAT_MIRROR, (0, 0, 0), (0.95, 0.95, 0.95), ior_n=0.25, ior_k=3.0),   # 3 conductor
        material(MAT_MIRROR, (0.3, 0.3, 0.35), (0.9, 0.9, 0.9), ior_n=1.5),     # 4 dielectric over Lambert
        material(MAT_MIRROR, (0.5, 0.45, 0.2), (0, 0, 0), ior_n=0.25, ior_k=3.0),   # 5 zero reflectance
        material(MAT_GLOW, (20.0, 20.0, 20.0)),                                 # 6 sphere light
    ])
    v, tris, tri_mat = _cornell_walls()
    spheres = np.zeros(3, SPHERE_DTYPE)
    spheres[0] = ((0.3, 0.3, 0.62), 0.3, 3)
    spheres[1] = ((0.72, 0.2, 0.33), 0.2, 0)
    spheres[2] = ((0.5, 0.86, 0.45), 0.07, 6)
    tripars = np.zeros(2, TRIPAR_DTYPE)
    tripars[0] = ((0.55, 0.3, 0.995), (0.3, 0, 0), (0, 0.45, 0), 1, 4)     # on the back wall
    tripars[1] = ((0.005, 0.45, 0.15), (0, 0, 0.3), (0, 0.3, 0), 1, 5)     # on the left wall
    pl = np.zeros(1, PLIGHT_DTYPE)
    pl[0] = ((0.5, 0.95, 0.2), (0.5, 0.5, 0.45), 2 * math.pi, 0.0, (0, 0, 1))   # omni
    return SceneData(materials=mats, vertices=v, triangles=tris, tri_mat=tri_mat, spheres=spheres,
                     tripars=tripars, point_lights=pl, name="mirror")


def mirror_params(width=64, height=64, spp=16, seed=0):
    return RenderParams(width=width, height=height, spp=spp, min_path_len=3, max_path_len=8,
                        direct_samples=1, seed=seed)


# An open scene (y up) lit only by lights that are not surfaces: a spotlight
# with a fringe (light/point-light.h:42-47, 67-83), a far light of angle 0
# (an infinitely distant point light, light/far-light.h:35-45) and a far
# light of non-zero angle (cone sampling, light/far-light.cc:96-156, which
# also appears as background).  Floor, Cook-Torrance, conductor Mirror and
# Lambert spheres.

def spot_far_scene():
    mats = _mats([
        material(MAT_LAMBERT, (0.6, 0.6, 0.6)),
        material(MAT_COOK_TORRANCE, (0.6, 0.3, 0.2), (1, 1, 1), m=0.15, ior_n=1.5),
        material(MAT_MIRROR, (0, 0, 0), (1, 1, 1), ior_n=0.25, ior_k=3.0),
        material(MAT_LAMBERT, (0.3, 0.5, 0.7)),
    ])
    v = np.array([[-1, 0, -1], [2, 0, -1], [2, 0, 2], [-1, 0, 2]], np.float32)
    tris = np.array([[0, 2, 1], [0, 3, 2]], np.uint32)
    spheres = np.zeros(3, SPHERE_DTYPE)
    spheres[0] = ((0.2, 0.25, 0.5), 0.25, 1)
    spheres[1] = ((0.75, 0.2, 0.45), 0.2, 2)
    spheres[2] = ((0.5, 0.15, 0.9), 0.15, 3)
    pl = np.zeros(1, PLIGHT_DTYPE)
    pl[0] = ((0.5, 1.5, 0.4), (3.0, 3.0, 2.8), math.radians(50.0), math.radians(15.0), (0, -1, 0))
    fl = np.zeros(2, FLIGHT_DTYPE)
    d0 = np.array([0.4, 0.8, -0.45])
    d1 = np.array([-0.5, 0.6, 0.3])
    fl[0] = (d0 / np.linalg.norm(d0), 0.0, (0.8, 0.75, 0.6))
    fl[1] = (d1 / np.linalg.norm(d1), math.radians(8.0), (40.0, 42.0, 48.0))
    return SceneData(materials=mats, vertices=v, triangles=tris, tri_mat=np.zeros(2, np.uint32),
                     spheres=spheres, point_lights=pl, far_lights=fl, name="spot_far")


def spot_far_camera(width, height):
    cam = Camera()
    cam.move((0.5, 0.9, -1.3))
    cam.point((0.5, 0.2, 0.5), (0, 1, 0))
    cam.set_vert_fov(math.radians(45.0), width / height)
    return cam


# Four concentric Glass spheres of different media in the Cornell box: a
# path inside the innermost one has four media on its stack
# (material/media.cc:76-118).

def nested_glass_scene():
    mats = _mats([
        material(MAT_LAMBERT, (0.73, 0.73, 0.73)),
        material(MAT_LAMBERT, (0.65, 0.05, 0.05)),
        material(MAT_LAMBERT, (0.12, 0.45, 0.15)),
        material(MAT_GLASS, ior_n=1.3),
        material(MAT_GLASS, ior_n=1.5, absorb=(0.4, 0.1, 0.05)),
        material(MAT_GLASS, ior_n=1.7),
        material(MAT_GLASS, ior_n=1.9, absorb=(0.05, 0.3, 0.6)),
        material(MAT_GLOW, (15.0, 15.0, 15.0)),
    ])
    v, tris, tri_mat = _cornell_walls()
    spheres = np.zeros(4, SPHERE_DTYPE)
    for k, r in enumerate((0.32, 0.24, 0.16, 0.08)):
        spheres[k] = ((0.5, 0.35, 0.5), r, 3 + k)
    tripars = np.zeros(1, TRIPAR_DTYPE)
    tripars[0] = ((0.375, 0.999, 0.375), (0, 0, 0.25), (0.25, 0, 0), 1, 7)
    return SceneData(materials=mats, vertices=v, triangles=tris, tri_mat=tri_mat, spheres=spheres,
                     tripars=tripars, name="nested_glass")


def nested_glass_params(width=64, height=64, spp=16, seed=0):
    return RenderParams(width=width, height=height, spp=spp, min_path_len=3, max_path_len=14,
                        direct_samples=1, seed=seed)


# ---------------------------------------------------------------------------
# Meshes as a PLY file gives them: right-handed (geometric normal e1 x e2),
# optionally with vertex normals.  A UV sphere of radius 0.3 resting on a
# floor quad, lit by a 0.5 x 0.5 area light; y up.

def _uv_sphere(center, r, n_lng, n_lat):
    """Vertices, outward unit normals and right-handed (counter-clockwise
    seen from outside) triangles of a UV sphere."""
    verts, nrms = [], []
    for i in range(n_lat + 1):
        th = math.pi * i / n_lat
        for j in range(n_lng):
            ph = 2 * math.pi * j / n_lng
            n = (math.sin(th) * math.cos(ph), math.cos(th), math.sin(th) * math.sin(ph))
            nrms.append(n)
            verts.append(tuple(c + r * x for c, x in zip(center, n)))
    tris = []
    for i in range(n_lat):
        for j in range(n_lng):
            a, b = i * n_lng + j, i * n_lng + (j + 1) % n_lng
            c, d = a + n_lng, b + n_lng
            if i > 0:
                tris.append([a, b, c])
            if i < n_lat - 1:
                tris.append([b, d, c])
    return np.array(verts), np.array(nrms), tris


def mesh_scene(smooth=True):
    """SMOOTH: the sphere (Cook-Torrance) and floor (Lambert) carry vertex
    normals.  Otherwise flat shading, the sphere is Glass and an emissive quad
    faces the camera: both depend on which side the right-handed normal is."""
    sv, sn, st = _uv_sphere((0.5, 0.3, 0.55), 0.3, 24, 12)
    fv = np.array([[-0.5, 0, -0.5], [1.5, 0, -0.5], [1.5, 0, 1.5], [-0.5, 0, 1.5]])
    fn = np.tile([[0.0, 1.0, 0.0]], (4, 1))
    base = len(sv)
    floor = [[base, base + 3, base + 2], [base, base + 2, base + 1]]   # e1 x e2 = +y
    verts, nrms = [sv, fv], [sn, fn]
    if smooth:
        mats = _mats([material(MAT_LAMBERT, (0.6, 0.6, 0.6)),
                      material(MAT_COOK_TORRANCE, (0.7, 0.3, 0.2), (1, 1, 1), m=0.2, ior_n=1.5),
                      material(MAT_GLOW, (10.0, 10.0, 10.0))])
        tris = floor + st
        tri_mat = [0, 0] + [1] * len(st)
    else:
        mats = _mats([material(MAT_LAMBERT, (0.6, 0.6, 0.6)),
                      material(MAT_GLASS, ior_n=1.5),
                      material(MAT_GLOW, (4.0, 3.0, 2.0)),
                      material(MAT_GLOW, (10.0, 10.0, 10.0))])
        qb = base + 4
        qv = np.array([[-0.2, 0.1, 0.9], [0.1, 0.1, 0.9], [0.1, 0.6, 0.9], [-0.2, 0.6, 0.9]])
        verts.append(qv)
        nrms.append(np.tile([[0.0, 0.0, -1.0]], (4, 1)))
        quad = [[qb, qb + 2, qb + 1], [qb, qb + 3, qb + 2]]   # e1 x e2 = -z, towards the camera
        tris = floor + st + quad
        tri_mat = [0, 0] + [1] * len(st) + [2, 2]
    tripars = np.zeros(1, TRIPAR_DTYPE)
    tripars[0] = ((0.25, 1.2, 0.25), (0, 0, 0.5), (0.5, 0, 0), 1, len(mats) - 1)   # e2 x e1 = -y
    v = np.concatenate(verts).astype(np.float32)
    n = np.concatenate(nrms).astype(np.float32)
    return SceneData(materials=mats, vertices=v, triangles=np.array(tris, np.uint32),
                     tri_mat=np.array(tri_mat, np.uint32), tripars=tripars,
                     normals=n if smooth else None, right_handed=True,
                     name="mesh_smooth" if smooth else "mesh_flat")


def mesh_camera(width, height):
    cam = Camera()
    cam.move((0.5, 0.55, -1.3))
    cam.point((0.5, 0.3, 0.5), (0, 1, 0))
    cam.set_vert_fov(math.radians(45.0), width / height)
    return cam


def mesh_params(width=64, height=64, spp=16, seed=0):
    return RenderParams(width=width, height=height, spp=spp, min_path_len=3, max_path_len=8,
                        direct_samples=1, seed=seed)


# ---------------------------------------------------------------------------
# Random triangle soup: centroids U[0,1]^3, edge lengths U(lo, hi), random
# orientation.

def _random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    r = np.empty((n, 3, 3))
    r[:, 0, 0] = 1 - 2 * (y * y + z * z); r[:, 0, 1] = 2 * (x * y - z * w); r[:, 0, 2] = 2 * (x * z + y * w)
    r[:, 1, 0] = 2 * (x * y + z * w); r[:, 1, 1] = 1 - 2 * (x * x + z * z); r[:, 1, 2] = 2 * (y * z - x * w)
    r[:, 2, 0] = 2 * (x * z - y * w); r[:, 2, 1] = 2 * (y * z + x * w); r[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return r


def random_triangles(n, seed=2, edge_lo=0.002, edge_hi=0.02, mats=None):
    """n random triangles as one mesh of one part (material 0)."""
    rng = np.random.default_rng(seed)
    cent = rng.uniform(0, 1, size=(n, 3))
    # Two edges from the first vertex, lengths U(lo, hi), at a random angle in
    # the triangle's plane, then a random rotation.
    l1 = rng.uniform(edge_lo, edge_hi, n)
    l2 = rng.uniform(edge_lo, edge_hi, n)
    ang = rng.uniform(0.3, math.pi - 0.3, n)
    e1 = np.stack([l1, np.zeros(n), np.zeros(n)], 1)
    e2 = np.stack([l2 * np.cos(ang), l2 * np.sin(ang), np.zeros(n)], 1)
    rot = _random_rotations(rng, n)
    e1 = np.einsum("nij,nj->ni", rot, e1)
    e2 = np.einsum("nij,nj->ni", rot, e2)
    v0 = cent - (e1 + e2) / 3
    verts = np.stack([v0, v0 + e1, v0 + e2], 1).reshape(-1, 3).astype(np.float32)
    tris = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    if mats is None:
        mats = _mats([material(MAT_LAMBERT, (0.7, 0.7, 0.7))])
    return SceneData(materials=mats, vertices=verts, triangles=tris,
                     tri_mat=np.zeros(n, np.uint32), name=f"soup{n}")


def random_rays(n, seed=3, lo=-0.1, hi=1.1):
    """Ray batch: origins U[lo,hi]^3, directions uniform on the sphere, t_max=inf.
    Returns (n, 7) float32 SoA rows ox oy oz dx dy dz tmax as a (7, n) array."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3))
    z = rng.uniform(-1, 1, n)
    phi = rng.uniform(0, 2 * math.pi, n)
    r = np.sqrt(np.maximum(0, 1 - z * z))
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    soa = np.empty((7, n), np.float32)
    soa[0:3] = o.T
    soa[3:6] = d.T
    soa[6] = np.inf
    return soa


def mixed_scene(n_tris, n_spheres, n_tripars, seed=5):
    """Random triangles, spheres (radius U(0.005, 0.05)) and tripars (edge
    lengths U(0.01, 0.1), half of them parallelograms) in the unit cube."""
    rng = np.random.default_rng(seed + 1000)
    s = random_triangles(n_tris, seed=seed)
    sph = np.zeros(n_spheres, SPHERE_DTYPE)
    sph["center"] = rng.uniform(0, 1, (n_spheres, 3))
    sph["radius"] = rng.uniform(0.005, 0.05, n_spheres)
    tp = np.zeros(n_tripars, TRIPAR_DTYPE)
    v0 = rng.uniform(0, 1, (n_tripars, 3))
    rot = _random_rotations(rng, n_tripars)
    e1 = np.einsum("nij,nj->ni", rot, np.stack([rng.uniform(0.01, 0.1, n_tripars),
                                                np.zeros(n_tripars), np.zeros(n_tripars)], 1))
    e2 = np.einsum("nij,nj->ni", rot, np.stack([np.zeros(n_tripars),
                                                rng.uniform(0.01, 0.1, n_tripars),
                                                np.zeros(n_tripars)], 1))
    tp["v0"], tp["e1"], tp["e2"] = v0, e1, e2
    tp["parallelogram"] = np.arange(n_tripars) % 2
    s.spheres, s.tripars = sph, tp
    s.name = f"mixed{n_tris}_{n_spheres}_{n_tripars}_s{seed}"
    return s


def scene_digest(sd):
    """sha256 over every array of a SceneData (pins fixtures to the exact
    float32 bits the generator produced)."""
    import hashlib
    h = hashlib.sha256()
    for a in (sd.materials, sd.vertices, sd.triangles, sd.tri_mat, sd.spheres, sd.tripars,
              sd.point_lights, sd.far_lights):
        h.update(np.ascontiguousarray(a).tobytes())
    if sd.envmap is not None:
        h.update(np.ascontiguousarray(sd.envmap).tobytes())
    if sd.normals is not None:
        h.update(np.ascontiguousarray(sd.normals).tobytes())
    if sd.right_handed:
        h.update(b"right-handed")
    return h.hexdigest()


# ---------------------------------------------------------------------------
# Terrain + spheres + procedural sky (z up).

def _value_noise(rng, res, x, y):
    g = rng.uniform(-1, 1, size=(res + 1, res + 1))
    xs, ys = x * res, y * res
    xi = np.clip(np.floor(xs).astype(int), 0, res - 1)
    yi = np.clip(np.floor(ys).astype(int), 0, res - 1)
    fx, fy = xs - xi, ys - yi
    sx, sy = fx * fx * (3 - 2 * fx), fy * fy * (3 - 2 * fy)
    a = g[xi, yi] * (1 - sx) + g[xi + 1, yi] * sx
    b = g[xi, yi + 1] * (1 - sx) + g[xi + 1, yi + 1] * sx
    return a * (1 - sy) + b * sy


def fbm_heightfield(n, seed=7, octaves=6, amplitude=0.2):
    rng = np.random.default_rng(seed)
    u = np.linspace(0, 1, n)
    x, y = np.meshgrid(u, u, indexing="ij")
    h = np.zeros((n, n))
    amp, freq, norm = 1.0, 4, 0.0
    for _ in range(octaves):
        h += amp * _value_noise(rng, freq, x, y)
        norm += amp
        amp *= 0.5
        freq *= 2
    return (amplitude * h / norm).astype(np.float32)


def sky_envmap(w=1024, h=512, sun_elev_deg=35.0, sun_azim_deg=40.0, sigma_deg=1.0, peak=5e3):
    """Lat-long sky (z up): vertical gradient plus a Gaussian sun."""
    v = (np.arange(h) + 0.5) / h
    lat = (0.5 - v) * math.pi                      # row 0 = top = zenith
    u = (np.arange(w) + 0.5) / w
    lng = (u - 0.5) * 2 * math.pi
    lat2, lng2 = np.meshgrid(lat, lng, indexing="ij")
    # Direction for (lat, lng) in the reference's z-axis lat-long convention
    # (geometry/spherical-coords.h:157-168): x = cos(lng) cos(lat),
    # y = -sin(lng) cos(lat), z = sin(lat).
    d = np.stack([np.cos(lng2) * np.cos(lat2), -np.sin(lng2) * np.cos(lat2), np.sin(lat2)], -1)
    t = np.clip(np.sin(lat2), 0, 1)[..., None]
    zenith = np.array([0.25, 0.45, 0.95])
    horizon = np.array([0.85, 0.9, 1.0])
    ground = np.array([0.25, 0.22, 0.2])
    sky = np.where(lat2[..., None] >= 0, horizon * (1 - t) + zenith * t, ground)
    se, sa = math.radians(sun_elev_deg), math.radians(sun_azim_deg)
    sdir = np.array([math.cos(sa) * math.cos(se), -math.sin(sa) * math.cos(se), math.sin(se)])
    ang = np.arccos(np.clip(d @ sdir, -1, 1))
    sig = math.radians(sigma_deg)
    sun = peak * np.exp(-0.5 * (ang / sig) ** 2)
    img = sky + sun[..., None] * np.array([1.0, 0.95, 0.85])
    return img.astype(np.float32)


def terrain_scene(n=1024, n_spheres=200, seed=11, env_w=1024, env_h=512):
    rng = np.random.default_rng(seed)
    hf = fbm_heightfield(n, seed=seed)
    u = np.linspace(0, 1, n, dtype=np.float32)
    x, y = np.meshgrid(u, u, indexing="ij")
    verts = np.stack([x, y, hf], -1).reshape(-1, 3).astype(np.float32)
    i, j = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    a = (i * n + j).ravel()
    b, c, d = a + n, a + n + 1, a + 1
    # Counter-clockwise seen from +z; the reference's meshes are left-handed
    # by default (normal = e2 x e1, surface/mesh.h:55), which is harmless for
    # shading since frames are flipped to face the viewer.
    tris = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)]).astype(np.uint32)
    recs = [material(MAT_LAMBERT, (0.45, 0.4, 0.33))]
    sph = np.zeros(n_spheres, SPHERE_DTYPE)
    kinds = rng.choice(3, size=n_spheres, p=[0.6, 0.2, 0.2])
    for k in range(n_spheres):
        r = rng.uniform(0.01, 0.05)
        px, py = rng.uniform(0.05, 0.95, 2)
        gx, gy = int(px * (n - 1)), int(py * (n - 1))
        pz = hf[gx, gy] + r + rng.uniform(0.0, 0.05)
        col = rng.uniform(0.2, 0.9, 3)
        if kinds[k] == 0:
            recs.append(material(MAT_COOK_TORRANCE, col, (1, 1, 1), m=rng.uniform(0.05, 0.5),
                                 ior_n=1.5))
        elif kinds[k] == 1:
            recs.append(material(MAT_GLASS, ior_n=1.5))
        else:
            recs.append(material(MAT_LAMBERT, col))
        sph[k] = ((px, py, pz), r, len(recs) - 1)
    env = sky_envmap(env_w, env_h)
    return SceneData(materials=_mats(recs), vertices=verts, triangles=tris,
                     tri_mat=np.zeros(len(tris), np.uint32), spheres=sph, envmap=env,
                     name=f"terrain{n}")


def terrain_camera(width, height):
    cam = Camera()
    cam.move((-0.35, -0.3, 0.45))
    cam.point((0.55, 0.55, 0.0), (0, 0, 1))
    cam.set_vert_fov(math.radians(45.0), width / height)
    return cam


def terrain_params(width=1920, height=1080, spp=64, seed=0):
    return RenderParams(width=width, height=height, spp=spp, min_path_len=3, max_path_len=16,
                        direct_samples=1, seed=seed)


# ---------------------------------------------------------------------------
# Random-soup scene with mixed materials and one area light, for the batched
# and served workloads.

def soup_scene(n_tris, seed, envmap=None, area_light=True):
    rng = np.random.default_rng(seed)
    recs = [material(MAT_LAMBERT, rng.uniform(0.2, 0.8, 3)),
            material(MAT_COOK_TORRANCE, rng.uniform(0.2, 0.8, 3), (1, 1, 1),
                     m=rng.uniform(0.05, 0.5), ior_n=1.5),
            material(MAT_GLOW, (12.0, 12.0, 12.0))]
    s = random_triangles(n_tris, seed=seed, mats=_mats(recs))
    # Lambert/Cook-Torrance mix: parts must be contiguous runs.
    n_ct = int(rng.uniform(0.2, 0.8) * n_tris)
    s.tri_mat = np.concatenate([np.zeros(n_tris - n_ct, np.uint32), np.ones(n_ct, np.uint32)])
    if area_light or envmap is None:
        tp = np.zeros(1, TRIPAR_DTYPE)
        tp[0] = ((0.35, 0.35, 1.3), (0.3, 0, 0), (0, 0.3, 0), 1, 2)   # faces -z
        s.tripars = tp
    if envmap is not None:
        s.envmap = envmap
    s.name = f"soup{n_tris}_s{seed}"
    return s


def orbit_camera(width, height, rng, center=(0.5, 0.5, 0.5), dist=1.8):
    z = rng.uniform(-0.6, 0.8)
    phi = rng.uniform(0, 2 * math.pi)
    r = math.sqrt(1 - z * z)
    pos = np.array(center) + dist * np.array([r * math.cos(phi), r * math.sin(phi), z])
    cam = Camera()
    cam.move(pos)
    cam.point(center, (0, 0, 1))
    cam.set_vert_fov(math.radians(50.0), width / height)
    return cam


# ---------------------------------------------------------------------------
# Batched workload: many independent small scenes of uneven size rendered
# together (1024 random-triangle soups of 1k-50k triangles, log-uniform, a
# Lambert/Cook-Torrance mix and one area light each; resolution from
# {64, 128, 256}^2, spp from {4, 16, 64}).

BATCH_RES = (64, 128, 256)
BATCH_SPP = (4, 16, 64)


def batch_workload(n_jobs=1024, seed=4, tri_lo=1000, tri_hi=50000):
    """[(SceneData, Camera, RenderParams)] for the batched workload."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n_jobs):
        n = int(round(math.exp(rng.uniform(math.log(tri_lo), math.log(tri_hi)))))
        res = int(rng.choice(BATCH_RES))
        spp = int(rng.choice(BATCH_SPP))
        sd = soup_scene(n, seed=10000 + k)
        cam = orbit_camera(res, res, rng)
        jobs.append((sd, cam, RenderParams(res, res, spp, seed=k)))
    return jobs


# ---------------------------------------------------------------------------
# Serving workload: 8 resident scenes of 10k-8M random triangles (mixed
# materials; area light, or a sky envmap for every other scene) and a stream
# of requests at Poisson arrivals, each a random scene, a camera on a sphere
# around it, a resolution from {128, 256, 512, 1024}^2 and spp from {4, 16, 64}.

SERVE_SIZES = (10_000, 50_000, 200_000, 1_000_000, 2_000_000, 4_000_000, 6_000_000, 8_000_000)
SERVE_RES = (128, 256, 512, 1024)
SERVE_SPP = (4, 16, 64)


def serve_scenes(sizes=SERVE_SIZES, seed=21):
    env = sky_envmap(256, 128, sigma_deg=3.0, peak=200.0)
    out = []
    for k, n in enumerate(sizes):
        if k % 2:
            out.append(soup_scene(n, seed=seed + k, envmap=env, area_light=False))
        else:
            out.append(soup_scene(n, seed=seed + k))
    return out


@dataclass
class Request:
    arrival_s: float
    scene: int
    camera: Camera
    params: RenderParams


def serve_requests(n=2000, rate=200.0, n_scenes=len(SERVE_SIZES), seed=22,
                   res_choices=SERVE_RES, spp_choices=SERVE_SPP):
    """N requests with exponential inter-arrival times at RATE per second."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    t -= t[0]
    reqs = []
    for k in range(n):
        res = int(rng.choice(res_choices))
        spp = int(rng.choice(spp_choices))
        sc = int(rng.integers(n_scenes))
        cam = orbit_camera(res, res, rng)
        reqs.append(Request(float(t[k]), sc, cam, RenderParams(res, res, spp, seed=k)))
    return reqs
