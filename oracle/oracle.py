"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle and the compiled reference.

* liblgoracle.so (oracle/lgoracle.c) -- this project's plain-C restatement of
  the reference BVH build and trace code, with ray counters.
* _ref/libref.so (oracle/ref_harness.cu) -- the reference's own sources
  (src/bvh.cpp, src/scene_loader.cpp, src/pathtracer.cu) compiled here: the
  host trace functions for the CPU, the reference kernels for the GPU.

Imported only by tests/, __graft_entry__.smoke() and bench.py (CPU baseline /
reference arm).  Never imported by the product package.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_LIB = HERE / "build" / "liblgoracle.so"
REF_LIB = HERE / "_ref" / "libref.so"

TRI_DTYPE = np.dtype([("v", "<f4", (3, 3)), ("n", "<f4", (3, 3)), ("uv", "<f4", (3, 2)), ("material", "<i4")])
NODE_DTYPE = np.dtype([("bbMin", "<f4", (3,)), ("bbMax", "<f4", (3,)), ("left", "<i4"), ("right", "<i4"),
                       ("firstTri", "<i4"), ("triCount", "<i4")])
POINT_DTYPE = np.dtype([("pos", "<f4", (3,)), ("color", "<f4", (3,)), ("intensity", "<f4"), ("radius", "<f4")])
DIR_DTYPE = np.dtype([("dir", "<f4", (3,)), ("color", "<f4", (3,)), ("intensity", "<f4")])


class CameraDesc(C.Structure):
    # Same layout as the reference CameraDesc and lg_camera.
    _fields_ = [("pos", C.c_float * 3), ("m", C.c_float * 16), ("fov", C.c_float), ("aspect", C.c_float),
                ("near", C.c_float), ("far", C.c_float), ("w", C.c_int32), ("h", C.c_int32)]


class Counters(C.Structure):
    _fields_ = [("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("node_visits", C.c_uint64),
                ("tri_tests", C.c_uint64)]


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def cam_desc(camera) -> CameraDesc:
    c = CameraDesc()
    c.pos[:] = [float(x) for x in camera.pos]
    c.m[:] = [float(x) for x in camera.camera_to_world]
    c.fov, c.aspect, c.near, c.far = camera.fov_y_deg, camera.aspect, camera.near_z, camera.far_z
    c.w, c.h = int(camera.width), int(camera.height)
    return c


def _sun(scene) -> np.ndarray:
    s = np.zeros(1, DIR_DTYPE)
    s[0] = scene.sun
    return s


_olib = None
_rlib = None


def olib():
    global _olib
    if _olib is None:
        if not ORACLE_LIB.exists():
            raise RuntimeError(f"{ORACLE_LIB} missing: run `make -C {HERE} oracle`")
        _olib = C.CDLL(str(ORACLE_LIB))
        _olib.lgo_build_bvh.restype = C.c_int
        _olib.lgo_render.restype = C.c_int
    return _olib


def ref_available() -> bool:
    return REF_LIB.exists()


def rlib():
    global _rlib
    if _rlib is None:
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} missing: run `make -C {HERE} ref` where the reference checkout exists")
        _rlib = C.CDLL(str(REF_LIB))
        _rlib.ref_scene_load.restype = C.c_void_p
        _rlib.ref_scene_load.argtypes = [C.c_char_p]
        _rlib.ref_scene_counts.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4
        _rlib.ref_scene_get.argtypes = [C.c_void_p] + [C.c_void_p] * 7
        _rlib.ref_scene_free.argtypes = [C.c_void_p]
        _rlib.ref_build_bvh.restype = C.c_int
        _rlib.ref_render_gpu.restype = C.c_int
        _rlib.ref_trace_cpu.restype = C.c_int
        _rlib.ref_omp_max_threads.restype = C.c_int
    return _rlib


# ---- oracle (restatement) ----
def oracle_build_bvh(tris: np.ndarray):
    """Returns (nodes, sorted triangles, perm, sorted codes)."""
    tris = np.ascontiguousarray(tris, TRI_DTYPE)
    n = len(tris)
    nodes = np.zeros(max(2 * n - 1, 1), NODE_DTYPE)
    out = np.zeros_like(tris)
    perm = np.zeros(max(n, 1), np.int32)
    codes = np.zeros(max(n, 1), np.uint32)
    cnt = olib().lgo_build_bvh(_p(tris), n, _p(nodes), _p(perm), _p(out), _p(codes))
    return nodes[:cnt].copy(), out, perm[:n].copy(), codes[:n].copy()


def oracle_render(scene, nodes, tris, spp, bounces, row_start=0, row_step=1, threads=0, camera=None):
    """Per-pixel accumulate of the restated reference; returns (accum (H,W,3) f32, counters dict)."""
    cam = camera if camera is not None else scene.camera
    acc = np.zeros((int(cam.height), int(cam.width), 3), np.float32)
    cnt = Counters()
    c = cam_desc(cam)
    sun = _sun(scene)
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    tris = np.ascontiguousarray(tris, TRI_DTYPE)
    alb = np.ascontiguousarray(scene.mat_albedo, np.float32)
    pts = np.ascontiguousarray(scene.points, POINT_DTYPE)
    rc = olib().lgo_render(_p(nodes), _p(tris), _p(alb), len(alb), _p(pts), len(pts), _p(sun), C.byref(c), spp,
                           bounces, row_start, row_step, threads, _p(acc), C.byref(cnt))
    assert rc == 0
    return acc, {"closest_rays": cnt.closest_rays, "shadow_rays": cnt.shadow_rays,
                 "node_visits": cnt.node_visits, "tri_tests": cnt.tri_tests}


def oracle_tonemap(accum: np.ndarray, spp: int) -> np.ndarray:
    a = np.ascontiguousarray(accum, np.float32)
    out = np.zeros(a.shape, np.uint8)
    inv = C.c_float(np.float32(1.0) / np.float32(spp))
    olib().lgo_tonemap(_p(a), _p(out), C.c_int(a.size // 3), inv)
    return out


# ---- reference (compiled sources) ----
def ref_build_bvh(tris: np.ndarray):
    """The reference BuildBVH; returns (nodes, reordered triangles)."""
    tris = np.ascontiguousarray(tris, TRI_DTYPE)
    n = len(tris)
    nodes = np.zeros(max(2 * n, 1), NODE_DTYPE)
    out = np.zeros_like(tris)
    cnt = C.c_int(0)
    rc = rlib().ref_build_bvh(_p(tris), n, _p(nodes), len(nodes), C.byref(cnt), _p(out))
    assert rc == 0
    return nodes[:cnt.value].copy(), out


def ref_load_scene(path: str):
    """The reference LoadSceneJSON; returns a dict of arrays or None on failure."""
    L = rlib()
    h = L.ref_scene_load(str(path).encode())
    if not h:
        return None
    try:
        nt, nm, npnt, nd = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        L.ref_scene_counts(h, C.byref(nt), C.byref(nm), C.byref(npnt), C.byref(nd))
        cam = CameraDesc()
        sun = np.zeros(1, DIR_DTYPE)
        tris = np.zeros(nt.value, TRI_DTYPE)
        alb = np.zeros((nm.value, 3), np.float32)
        emi = np.zeros((nm.value, 3), np.float32)
        pts = np.zeros(npnt.value, POINT_DTYPE)
        dirs = np.zeros(nd.value, DIR_DTYPE)
        L.ref_scene_get(h, C.addressof(cam), _p(sun), _p(tris), _p(alb), _p(emi), _p(pts), _p(dirs))
        return {"camera": cam, "sun": sun[0], "tris": tris, "albedo": alb, "emissive": emi, "points": pts,
                "directionals": dirs}
    finally:
        L.ref_scene_free(h)


def ref_trace_cpu(scene, nodes, tris, spp, bounces, row_start=0, row_step=1, threads=0, camera=None):
    """The reference's trace code on the host (OpenMP over rows); returns accum (H,W,3)."""
    cam = camera if camera is not None else scene.camera
    acc = np.zeros((int(cam.height), int(cam.width), 3), np.float32)
    c = cam_desc(cam)
    sun = _sun(scene)
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    tris = np.ascontiguousarray(tris, TRI_DTYPE)
    alb = np.ascontiguousarray(scene.mat_albedo, np.float32)
    emi = np.ascontiguousarray(scene.mat_emissive, np.float32)
    pts = np.ascontiguousarray(scene.points, POINT_DTYPE)
    rc = rlib().ref_trace_cpu(_p(nodes), _p(tris), _p(alb), _p(emi), len(alb), _p(pts), len(pts), _p(sun),
                              C.byref(c), spp, bounces, row_start, row_step, threads, _p(acc))
    assert rc == 0
    return acc


def ref_render_gpu(scene, nodes, tris, spp, bounces, camera=None, sorted_path=False):
    """The reference kernels on the GPU; returns (accum (H,W,3) f32, rgb (H,W,3) u8, kernel ms).
    sorted_path: its ray-sorted render (RenderSceneCUDASorted, pathtracer.cu:759-909) instead of
    accumulate_kernel."""
    cam = camera if camera is not None else scene.camera
    H, W = int(cam.height), int(cam.width)
    acc = np.zeros((H, W, 3), np.float32)
    rgb = np.zeros((H, W, 3), np.uint8)
    ms = C.c_float(0)
    c = cam_desc(cam)
    sun = _sun(scene)
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    tris = np.ascontiguousarray(tris, TRI_DTYPE)
    alb = np.ascontiguousarray(scene.mat_albedo, np.float32)
    emi = np.ascontiguousarray(scene.mat_emissive, np.float32)
    pts = np.ascontiguousarray(scene.points, POINT_DTYPE)
    fn = rlib().ref_render_sorted_gpu if sorted_path else rlib().ref_render_gpu
    rc = fn(_p(nodes), len(nodes), _p(tris), len(tris), _p(alb), _p(emi), len(alb), _p(pts),
            len(pts), _p(sun), C.byref(c), spp, bounces, _p(acc), _p(rgb), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU render failed with CUDA error {rc}")
    return acc, rgb, ms.value


def ref_omp_threads() -> int:
    return rlib().ref_omp_max_threads()


def ref_gbuffer_gpu(scene, nodes, tris, camera=None):
    """The reference gbuffer_kernel on the GPU; returns (albedo, normal, worldpos) (H,W,3) u8."""
    cam = camera if camera is not None else scene.camera
    H, W = int(cam.height), int(cam.width)
    out = [np.zeros((H, W, 3), np.uint8) for _ in range(3)]
    c = cam_desc(cam)
    sun = _sun(scene)
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    tris = np.ascontiguousarray(tris, TRI_DTYPE)
    alb = np.ascontiguousarray(scene.mat_albedo, np.float32)
    emi = np.ascontiguousarray(scene.mat_emissive, np.float32)
    pts = np.ascontiguousarray(scene.points, POINT_DTYPE)
    rc = rlib().ref_gbuffer_gpu(_p(nodes), len(nodes), _p(tris), len(tris), _p(alb), _p(emi), len(alb), _p(pts),
                                len(pts), _p(sun), C.byref(c), _p(out[0]), _p(out[1]), _p(out[2]))
    if rc != 0:
        raise RuntimeError(f"reference G-buffer failed with CUDA error {rc}")
    return tuple(out)


def ref_set_textures(paths):
    """Per-material texture files for ref_render_gpu / ref_gbuffer_gpu ('' or None: untextured)."""
    arr = (C.c_char_p * max(len(paths), 1))(*[(p or "").encode() for p in paths])
    rlib().ref_set_textures(len(paths), arr)


def ref_image_load(path):
    """stbi_load(path, 4 channels) as the reference uses it; returns (H,W,4) u8 or None."""
    L = rlib()
    w, h = C.c_int(), C.c_int()
    out = C.POINTER(C.c_uint8)()
    if L.ref_image_load(str(path).encode(), C.byref(w), C.byref(h), C.byref(out)) != 0:
        return None
    try:
        return np.ctypeslib.as_array(out, shape=(h.value, w.value, 4)).copy()
    finally:
        L.ref_image_free(out)
