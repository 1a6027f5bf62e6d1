"""Scenes as numpy record arrays, scene.json I/O through liblumina, and the
seeded procedural scenes used by the tests and the benchmark.

The record layouts are the reference's (include/scene.h): a triangle is
9 vertex floats, 9 normal floats, 6 uv floats and an int material (100 B).
Coordinates are Z-up, as the reference's camera override assumes
(main.cpp:40, worldUp = (0,0,1)).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np

from . import _ffi
from ._ffi import DIR_DTYPE, POINT_DTYPE, TRI_DTYPE, LgCamera, LgDirLight, LgSceneDesc, check, lib, ptr


@dataclasses.dataclass
class Camera:
    pos: np.ndarray  # (3,) f32
    camera_to_world: np.ndarray  # (16,) f32; rows 0/1/2 forward/left/up, row 3 position
    fov_y_deg: float = 60.0
    aspect: float = 1.0
    near_z: float = 0.1
    far_z: float = 1000.0
    width: int = 1920
    height: int = 1080

    def to_c(self) -> LgCamera:
        c = LgCamera()
        c.pos[:] = [float(x) for x in np.asarray(self.pos, np.float32)]
        c.camera_to_world[:] = [float(x) for x in np.asarray(self.camera_to_world, np.float32)]
        c.fov_y_deg, c.aspect, c.near_z, c.far_z = self.fov_y_deg, self.aspect, self.near_z, self.far_z
        c.width, c.height = int(self.width), int(self.height)
        return c

    @staticmethod
    def from_c(c: LgCamera) -> "Camera":
        return Camera(np.array(c.pos[:], np.float32), np.array(c.camera_to_world[:], np.float32), c.fov_y_deg,
                      c.aspect, c.near_z, c.far_z, c.width, c.height)

    def look_at(self, pos, target) -> "Camera":
        """overwrite_camera (reference main.cpp:29-59) through the C library."""
        c = self.to_c()
        p = (C.c_float * 3)(*[float(x) for x in pos])
        t = (C.c_float * 3)(*[float(x) for x in target])
        lib().lg_look_at(C.byref(c), p, t)
        return Camera.from_c(c)

    def copy(self) -> "Camera":
        return dataclasses.replace(self, pos=np.array(self.pos, np.float32),
                                   camera_to_world=np.array(self.camera_to_world, np.float32))


@dataclasses.dataclass
class Scene:
    camera: Camera
    sun: np.ndarray  # DIR_DTYPE scalar record
    tris: np.ndarray  # TRI_DTYPE (N,)
    mat_albedo: np.ndarray  # (M, 3) f32
    mat_emissive: np.ndarray  # (M, 3) f32
    points: np.ndarray  # POINT_DTYPE (P,)
    directionals: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, DIR_DTYPE))
    textures: list = dataclasses.field(default_factory=list)  # per material "diffuse_tex" ('' = none)

    def __post_init__(self):
        self.tris = np.ascontiguousarray(self.tris, TRI_DTYPE)
        self.mat_albedo = np.ascontiguousarray(self.mat_albedo, np.float32).reshape(-1, 3)
        self.mat_emissive = np.ascontiguousarray(self.mat_emissive, np.float32).reshape(-1, 3)
        self.points = np.ascontiguousarray(self.points, POINT_DTYPE)
        self.directionals = np.ascontiguousarray(self.directionals, DIR_DTYPE)

    @property
    def n_tris(self) -> int:
        return int(self.tris.shape[0])

    def desc(self) -> LgSceneDesc:
        """A C view of this scene (valid while the arrays live)."""
        d = LgSceneDesc()
        d.camera = self.camera.to_c()
        s = LgDirLight()
        s.dir[:] = [float(x) for x in self.sun["dir"]]
        s.color[:] = [float(x) for x in self.sun["color"]]
        s.intensity = float(self.sun["intensity"])
        d.sun = s
        d.tris, d.n_tris = ptr(self.tris), self.n_tris
        d.mat_albedo, d.mat_emissive, d.n_mats = ptr(self.mat_albedo), ptr(self.mat_emissive), len(self.mat_albedo)
        d.points, d.n_points = ptr(self.points), len(self.points)
        d.directionals, d.n_directionals = ptr(self.directionals), len(self.directionals)
        return d

    def _save(self, path: str, fn: str) -> None:
        h = C.c_void_p()
        d = self.desc()
        check(lib().lg_scene_create(C.byref(d), C.byref(h)))
        try:
            for m, t in enumerate(self.textures):
                if t:
                    check(lib().lg_scene_set_texture(h, m, str(t).encode()))
            check(getattr(lib(), fn)(h, str(path).encode()))
        finally:
            lib().lg_scene_destroy(h)

    def save_json(self, path: str) -> None:
        """scene.json in the reference schema (scene_loader.cpp:26-138)."""
        self._save(path, "lg_scene_save_json")

    def save_bin(self, path: str) -> None:
        """Binary scene file (same content; loads without text parsing)."""
        self._save(path, "lg_scene_save_bin")

    @staticmethod
    def load_json(path: str, verbose: bool = False, threads: int = 0) -> "Scene":
        """LoadSceneJSON (reference scene_loader.cpp:26-138) through the C library;
        binary scene files are recognised and loaded too."""
        h = C.c_void_p()
        check(lib().lg_scene_load_json(str(path).encode(), 1 if verbose else 0, threads, C.byref(h)))
        try:
            d = LgSceneDesc()
            check(lib().lg_scene_describe(h, C.byref(d)))
            sc = Scene._from_desc(d)
            sc.textures = [lib().lg_scene_texture(h, m).decode() for m in range(d.n_mats)]
            return sc
        finally:
            lib().lg_scene_destroy(h)

    @staticmethod
    def _from_desc(d: LgSceneDesc) -> "Scene":
        def arr(p, n, dtype, shape=None):
            if n == 0 or not p:
                return np.zeros((0,) + (shape or ()), dtype)
            nbytes = n * np.dtype(dtype).itemsize * (int(np.prod(shape)) if shape else 1)
            buf = (C.c_char * nbytes).from_address(p)
            a = np.frombuffer(buf, dtype=dtype).copy()
            return a.reshape((n,) + shape) if shape else a

        sun = np.zeros((), DIR_DTYPE)
        sun["dir"], sun["color"], sun["intensity"] = d.sun.dir[:], d.sun.color[:], d.sun.intensity
        return Scene(camera=Camera.from_c(d.camera), sun=sun, tris=arr(d.tris, d.n_tris, TRI_DTYPE),
                     mat_albedo=arr(d.mat_albedo, d.n_mats, np.float32, (3,)),
                     mat_emissive=arr(d.mat_emissive, d.n_mats, np.float32, (3,)),
                     points=arr(d.points, d.n_points, POINT_DTYPE),
                     directionals=arr(d.directionals, d.n_directionals, DIR_DTYPE))


# ---------------------------------------------------------------------------
# Procedural geometry (float64 construction, float32 records)
# ---------------------------------------------------------------------------
def icosphere(subdiv: int):
    """Unit icosphere: (vertices (V,3) f64, faces (F,3) i64), F = 20 * 4**subdiv."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        ab, bc, ca = (inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base)
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    return v, f


def grid_mesh(n: int, size: float, amp: float, rng: np.random.Generator):
    """n x n quads over [-size/2, size/2]^2, z displaced by a sum of sines; 2*n*n faces."""
    xs = np.linspace(-size / 2, size / 2, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    Z = np.zeros_like(X)
    dZx = np.zeros_like(X)
    dZy = np.zeros_like(X)
    for _ in range(4):
        fx, fy = rng.uniform(0.2, 1.5, 2) * (2 * math.pi / size) * 4
        px, py = rng.uniform(0, 2 * math.pi, 2)
        a = amp * rng.uniform(0.3, 1.0)
        Z += a * np.sin(fx * X + px) * np.cos(fy * Y + py)
        dZx += a * fx * np.cos(fx * X + px) * np.cos(fy * Y + py)
        dZy += -a * fy * np.sin(fx * X + px) * np.sin(fy * Y + py)
    v = np.stack([X, Y, Z], -1).reshape(-1, 3)
    nrm = np.stack([-dZx, -dZy, np.ones_like(Z)], -1).reshape(-1, 3)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    i, j = i.ravel(), j.ravel()
    v00, v10, v01, v11 = i * (n + 1) + j, (i + 1) * (n + 1) + j, i * (n + 1) + j + 1, (i + 1) * (n + 1) + j + 1
    f = np.concatenate([np.stack([v00, v10, v11], 1), np.stack([v00, v11, v01], 1)])
    uv = np.stack([(X / size + 0.5), (Y / size + 0.5)], -1).reshape(-1, 2)
    return v, nrm, f, uv


def box_mesh(half):
    """Axis-aligned box with outward flat normals: (v (36,3), n (36,3)) as 12 triangles."""
    hx, hy, hz = half
    c = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [hx, hy, -hz], [-hx, hy, -hz], [-hx, -hy, hz], [hx, -hy, hz],
                  [hx, hy, hz], [-hx, hy, hz]])
    quads = [([0, 3, 2, 1], [0, 0, -1]), ([4, 5, 6, 7], [0, 0, 1]), ([0, 1, 5, 4], [0, -1, 0]),
             ([2, 3, 7, 6], [0, 1, 0]), ([1, 2, 6, 5], [1, 0, 0]), ([3, 0, 4, 7], [-1, 0, 0])]
    tv, tn = [], []
    for q, nrm in quads:
        for tri in ([q[0], q[1], q[2]], [q[0], q[2], q[3]]):
            tv.append(c[tri])
            tn.append([nrm] * 3)
    return np.array(tv, np.float64), np.array(tn, np.float64)


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _tri_records(v, n, uv, material) -> np.ndarray:
    out = np.zeros(len(v), TRI_DTYPE)
    out["v"] = v.astype(np.float32)
    out["n"] = n.astype(np.float32)
    out["uv"] = uv.astype(np.float32)
    out["material"] = material
    return out


def _indexed(vert, nrm, uvs, faces, material):
    return _tri_records(vert[faces], nrm[faces], uvs[faces], material)


def _sphere_uv(v):
    return np.stack([np.arctan2(v[:, 1], v[:, 0]) / (2 * math.pi) + 0.5, np.arccos(np.clip(v[:, 2], -1, 1)) / math.pi],
                    -1)


def look_at_f32(pos, target, camera_to_world=None):
    """overwrite_camera (reference main.cpp:29-59) in float32 numpy, the same
    single-precision operations in the same order as lg_look_at, so the two
    agree bit for bit (checked by a test); lets the scene generators run
    without the CUDA library.  Returns (pos, camera_to_world) or None when
    |target - pos| < 1e-8 (the reference leaves the camera unchanged)."""
    f = np.float32
    p = np.asarray(pos, np.float32).reshape(3)
    t = np.asarray(target, np.float32).reshape(3)
    fx, fy, fz = f(t[0] - p[0]), f(t[1] - p[1]), f(t[2] - p[2])
    fl = np.sqrt(f(f(f(fx * fx) + f(fy * fy)) + f(fz * fz)))
    if fl < f(1e-8):
        return None
    fx, fy, fz = f(fx / fl), f(fy / fl), f(fz / fl)
    lx, ly, lz = f(-fy), fx, f(0.0)
    ll = np.sqrt(f(f(f(lx * lx) + f(ly * ly)) + f(lz * lz)))
    if ll < f(1e-6):
        lx, ly, lz, ll = f(0.0), f(1.0), f(0.0), f(1.0)
    lx, ly, lz = f(lx / ll), f(ly / ll), f(lz / ll)
    ux = f(f(fy * lz) - f(fz * ly))
    uy = f(f(fz * lx) - f(fx * lz))
    uz = f(f(fx * ly) - f(fy * lx))
    m = np.array(camera_to_world if camera_to_world is not None else np.eye(4).ravel(), np.float32).copy()
    m[0:4] = [fx, fy, fz, 0]
    m[4:8] = [lx, ly, lz, 0]
    m[8:12] = [ux, uy, uz, 0]
    m[12:16] = [p[0], p[1], p[2], 1]
    return p.copy(), m


def look_at_camera(pos, target, width, height, fov=60.0, aspect=None) -> Camera:
    """A pinhole camera at pos looking at target (overwrite_camera's frame)."""
    p, m = look_at_f32(pos, target)
    return Camera(p, m, fov, float(aspect if aspect is not None else width / height), 0.1, 1000.0, width, height)


def box_scene(seed: int = 1, width: int = 512, height: int = 256, sphere_subdiv: int = 4) -> Scene:
    """Small plain-method scene: 10 axis-aligned quads (a room plus four
    panels, 20 triangles) and 4 icospheres of 20*4**sphere_subdiv triangles
    (5,120 each at the default), per-mesh albedo U[0.1,0.9], one point light
    of intensity 50 in the upper half of the room, sun present with zero
    intensity, 60 degree fov, aspect 2."""
    rng = np.random.default_rng(seed)
    X, Y, Z = 4.0, 4.0, 4.0
    quads = [  # (corners ccw seen from the normal side, normal)
        ([[-X, -Y, 0], [X, -Y, 0], [X, Y, 0], [-X, Y, 0]], [0, 0, 1]),
        ([[-X, -Y, Z], [-X, Y, Z], [X, Y, Z], [X, -Y, Z]], [0, 0, -1]),
        ([[-X, -Y, 0], [-X, Y, 0], [-X, Y, Z], [-X, -Y, Z]], [1, 0, 0]),
        ([[X, -Y, 0], [X, -Y, Z], [X, Y, Z], [X, Y, 0]], [-1, 0, 0]),
        ([[-X, -Y, 0], [-X, -Y, Z], [X, -Y, Z], [X, -Y, 0]], [0, 1, 0]),
        ([[-X, Y, 0], [X, Y, 0], [X, Y, Z], [-X, Y, Z]], [0, -1, 0]),
        ([[1.0, -Y, 0], [1.0, -Y, 2.5], [1.0, -1.5, 2.5], [1.0, -1.5, 0]], [-1, 0, 0]),
        ([[-1.5, 1.5, 0], [-1.5, 1.5, 1.8], [-1.5, Y, 1.8], [-1.5, Y, 0]], [1, 0, 0]),
        ([[2.0, -1.0, 1.2], [3.5, -1.0, 1.2], [3.5, 1.0, 1.2], [2.0, 1.0, 1.2]], [0, 0, 1]),
        ([[-3.5, -3.5, 2.8], [-2.0, -3.5, 2.8], [-2.0, -2.0, 2.8], [-3.5, -2.0, 2.8]], [0, 0, 1]),
    ]
    recs = []
    for m, (q, nrm) in enumerate(quads):
        q = np.array(q, np.float64)
        v = np.array([[q[0], q[1], q[2]], [q[0], q[2], q[3]]])
        n = np.tile(np.array(nrm, np.float64), (2, 3, 1))
        uv = np.tile(np.array([[0, 0], [1, 0], [1, 1]], np.float64), (2, 1, 1))
        recs.append(_tri_records(v, n, uv, m))
    sv, sf = icosphere(sphere_subdiv)
    suv = _sphere_uv(sv)
    centers = [(-0.5, -2.0, 0.9), (2.6, 0.2, 2.0), (0.0, 1.8, 1.0), (-2.6, 1.0, 0.7)]
    for k, c in enumerate(centers):
        r = rng.uniform(0.6, 1.0)
        recs.append(_indexed(sv * r + np.array(c), sv, suv, sf, len(quads) + k))
    n_mats = len(quads) + len(centers)
    albedo = rng.uniform(0.1, 0.9, (n_mats, 3)).astype(np.float32)
    points = np.zeros(1, POINT_DTYPE)
    points["pos"] = [rng.uniform(-3, 3), rng.uniform(-3, 3), rng.uniform(Z / 2 + 0.5, Z - 0.3)]
    points["color"] = [1.0, 1.0, 1.0]
    points["intensity"] = 50.0
    points["radius"] = float(np.linalg.norm([2 * X, 2 * Y, Z]))
    sun = np.zeros((), DIR_DTYPE)
    sun["dir"], sun["color"], sun["intensity"] = [0.3, 0.2, -1.0], [1.0, 1.0, 1.0], 0.0
    cam = look_at_camera([-3.6, -0.4, 2.0], [1.0, 0.2, 1.2], width, height, 60.0, 2.0)
    return Scene(cam, sun, np.concatenate(recs), albedo, np.zeros_like(albedo), points)


ENGINE_CENTER = np.array([0.0, 0.0, 1.5])


def engine_scene(seed: int = 7, width: int = 1728, height: int = 864, grid_n: int = 256, n_grids: int = 7,
                 n_spheres: int = 26, sphere_subdiv: int = 4, n_boxes: int = 29) -> Scene:
    """Engine-scale plain-method scene: 62 meshes (7 noise-displaced 256x256
    grids of 131,072 triangles, 26 icospheres of 5,120, 29 boxes of 12;
    1,050,972 triangles at the defaults) under random similarity transforms in
    a 40 m box, albedo U[0.05,0.95], a sun and two point lights, 1728x864 at
    aspect 2.  Smaller variants (grid_n, counts) keep the same construction."""
    rng = np.random.default_rng(seed)
    recs = []
    mat = 0
    for g in range(n_grids):
        if g == 0:
            v, n, f, uv = grid_mesh(grid_n, 40.0, 0.35, rng)
            R, s, t = np.eye(3), 1.0, np.array([0.0, 0.0, 0.0])
        else:
            v, n, f, uv = grid_mesh(grid_n, rng.uniform(8, 16), rng.uniform(0.3, 1.2), rng)
            ang = rng.uniform(0, 2 * math.pi)
            tilt = rng.uniform(0.0, 1.2)
            Rz = np.array([[math.cos(ang), -math.sin(ang), 0], [math.sin(ang), math.cos(ang), 0], [0, 0, 1]])
            Rx = np.array([[1, 0, 0], [0, math.cos(tilt), -math.sin(tilt)], [0, math.sin(tilt), math.cos(tilt)]])
            R, s = Rz @ Rx, rng.uniform(0.8, 1.2)
            t = np.array([rng.uniform(-14, 14), rng.uniform(-14, 14), rng.uniform(1.0, 6.0)])
        recs.append(_indexed(v @ R.T * s + t, n @ R.T, uv, f, mat))
        mat += 1
    sv, sf = icosphere(sphere_subdiv)
    suv = _sphere_uv(sv)
    for _ in range(n_spheres):
        R, s = random_rotation(rng), rng.uniform(0.5, 2.5)
        t = np.array([rng.uniform(-17, 17), rng.uniform(-17, 17), rng.uniform(0.5, 9.0)])
        recs.append(_indexed(sv @ R.T * s + t, sv @ R.T, suv, sf, mat))
        mat += 1
    for _ in range(n_boxes):
        bv, bn = box_mesh(rng.uniform(0.25, 2.0, 3))
        R, s = random_rotation(rng), rng.uniform(0.8, 1.5)
        t = np.array([rng.uniform(-18, 18), rng.uniform(-18, 18), rng.uniform(0.5, 10.0)])
        uv = np.tile(np.array([[0, 0], [1, 0], [1, 1]], np.float64), (12, 1, 1))
        recs.append(_tri_records(bv @ R.T * s + t, bn @ R.T, uv, mat))
        mat += 1
    albedo = rng.uniform(0.05, 0.95, (mat, 3)).astype(np.float32)
    points = np.zeros(2, POINT_DTYPE)
    points["pos"] = [[-6.0, 4.0, 7.0], [8.0, -5.0, 5.0]]
    points["color"] = [[1.0, 0.9, 0.8], [0.8, 0.9, 1.0]]
    points["intensity"] = [30.0, 25.0]
    points["radius"] = [15.0, 12.0]
    sun = np.zeros((), DIR_DTYPE)
    d = np.array([-0.4, -0.3, -1.0])
    sun["dir"], sun["color"], sun["intensity"] = d / np.linalg.norm(d), [1.0, 0.95, 0.9], 2.5
    cam = look_at_camera([20.0, -6.0, 5.0], ENGINE_CENTER, width, height, 60.0, 2.0)
    return Scene(cam, sun, np.concatenate(recs), albedo, np.zeros_like(albedo), points)


def orbit_poses(n: int, seed: int = 11, center=ENGINE_CENTER):
    """Seeded orbit: radius U[15,25] m, height U[2,8] m, azimuth U[0,2pi), looking at the scene centre."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        a, r, h = rng.uniform(0, 2 * math.pi), rng.uniform(15, 25), rng.uniform(2, 8)
        out.append(((center[0] + r * math.cos(a), center[1] + r * math.sin(a), h), tuple(center)))
    return out
