"""ctypes binding of liblumina.so (include/lumina.h).

The shared library is built in-tree (``make -C luminagi-cudaref_b200``) and is
the only implementation: there is no Python or CPU fallback, and loading fails
loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent.parent
LIB_PATH = PKG_DIR / "lib" / "liblumina.so"
CLI_PATH = PKG_DIR / "bin" / "cuda_ref"

LG_OK = 0
LG_ERR_INVALID = -1
LG_ERR_CUDA = -2
LG_ERR_IO = -3
LG_ERR_PARSE = -4
LG_ERR_NOMEM = -5
LG_ERR_DEVICE = -6
LG_ERR_CAPACITY = -7
LG_RENDER_ACCUM64 = 1
LG_RENDER_NO_RAY_SORT = 2
LG_ISECT_MOLLER_TRUMBORE = 0
LG_ISECT_WATERTIGHT = 1
LG_UNET_RELU, LG_UNET_BILINEAR, LG_UNET_LOG_HDR, LG_UNET_HDR_VARIANT = 1, 2, 4, 7

# Record layouts (byte-identical to the reference's Triangle / BvhNode / lights).
TRI_DTYPE = np.dtype([("v", "<f4", (3, 3)), ("n", "<f4", (3, 3)), ("uv", "<f4", (3, 2)), ("material", "<i4")])
NODE_DTYPE = np.dtype([("bbMin", "<f4", (3,)), ("bbMax", "<f4", (3,)), ("left", "<i4"), ("right", "<i4"),
                       ("firstTri", "<i4"), ("triCount", "<i4")])
POINT_DTYPE = np.dtype([("pos", "<f4", (3,)), ("color", "<f4", (3,)), ("intensity", "<f4"), ("radius", "<f4")])
DIR_DTYPE = np.dtype([("dir", "<f4", (3,)), ("color", "<f4", (3,)), ("intensity", "<f4")])
assert TRI_DTYPE.itemsize == 100 and NODE_DTYPE.itemsize == 40
assert POINT_DTYPE.itemsize == 32 and DIR_DTYPE.itemsize == 28


class LgCamera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("camera_to_world", C.c_float * 16), ("fov_y_deg", C.c_float),
                ("aspect", C.c_float), ("near_z", C.c_float), ("far_z", C.c_float), ("width", C.c_int32),
                ("height", C.c_int32)]


class LgDirLight(C.Structure):
    _fields_ = [("dir", C.c_float * 3), ("color", C.c_float * 3), ("intensity", C.c_float)]


class LgSceneDesc(C.Structure):
    _fields_ = [("camera", LgCamera), ("sun", LgDirLight), ("tris", C.c_void_p), ("n_tris", C.c_int32),
                ("mat_albedo", C.c_void_p), ("mat_emissive", C.c_void_p), ("n_mats", C.c_int32),
                ("points", C.c_void_p), ("n_points", C.c_int32), ("directionals", C.c_void_p),
                ("n_directionals", C.c_int32)]


class LgRenderOpts(C.Structure):
    _fields_ = [("spp", C.c_int32), ("max_bounces", C.c_int32), ("sample_base", C.c_int32), ("flags", C.c_uint32)]


class LgRenderStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_float), ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("node_fetches", C.c_uint64), ("tri_tests", C.c_uint64), ("leaf_fetches", C.c_uint64)]


class LuminaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lumina error {code}: {msg}")
        self.code = code


# Every symbol include/lumina.h declares, with (restype, argtypes).
_P = C.c_void_p
_I = C.c_int
SIGNATURES = {
    "lg_last_error": (C.c_char_p, []),
    "lg_version": (_I, []),
    "lg_scene_load_json": (_I, [C.c_char_p, _I, _I, C.POINTER(_P)]),
    "lg_scene_create": (_I, [C.POINTER(LgSceneDesc), C.POINTER(_P)]),
    "lg_scene_describe": (_I, [_P, C.POINTER(LgSceneDesc)]),
    "lg_scene_set_camera": (_I, [_P, C.POINTER(LgCamera)]),
    "lg_scene_save_json": (_I, [_P, C.c_char_p]),
    "lg_scene_save_bin": (_I, [_P, C.c_char_p]),
    "lg_scene_texture": (C.c_char_p, [_P, _I]),
    "lg_scene_set_texture": (_I, [_P, _I, C.c_char_p]),
    "lg_scene_destroy": (None, [_P]),
    "lg_image_load": (_I, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.POINTER(C.c_uint8))]),
    "lg_image_free": (None, [C.POINTER(C.c_uint8)]),
    "lg_look_at": (None, [C.POINTER(LgCamera), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "lg_build_bvh": (_I, [_P, C.c_int32, _P, C.POINTER(C.c_int32), _P, _P]),
    "lg_build_bvh_device": (_I, [_P, C.c_int32, _P, C.POINTER(C.c_int32), _P, _P, _P]),
    "lg_build_bvh_device_noalloc": (_I, [_P, C.c_int32, _P, C.POINTER(C.c_int32), _P, _P, _P]),
    "lg_renderer_create": (_I, [_I, C.POINTER(_P)]),
    "lg_renderer_destroy": (None, [_P]),
    "lg_renderer_set_scene": (_I, [_P, C.POINTER(LgSceneDesc)]),
    "lg_renderer_set_scene_bvh": (_I, [_P, C.POINTER(LgSceneDesc), _P, C.c_int32]),
    "lg_renderer_get_bvh": (_I, [_P, _P, C.POINTER(C.c_int32), _P]),
    "lg_renderer_set_counting": (_I, [_P, _I]),
    "lg_renderer_set_bvh_width": (_I, [_P, _I]),
    "lg_renderer_set_intersection": (_I, [_P, _I]),
    "lg_renderer_set_render_tree": (_I, [_P, _I]),
    "lg_renderer_set_refill_threshold": (_I, [_P, _I]),
    "lg_renderer_get_refill_threshold": (_I, [_P]),
    "lg_renderer_set_leaf_quorum": (_I, [_P, _I]),
    "lg_renderer_get_leaf_quorum": (_I, [_P]),
    "lg_renderer_get_render_tree": (_I, [_P, C.POINTER(C.c_int32)]),
    "lg_renderer_autotune": (_I, [_P, C.POINTER(LgCamera), _I, _I, C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "lg_renderer_autotune_schedule": (_I, [_P, C.POINTER(LgCamera), _I, _I, C.POINTER(C.c_int32),
                                           C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "lg_renderer_set_texture": (_I, [_P, _I, _P, C.c_int32, C.c_int32]),
    "lg_renderer_load_textures": (_I, [_P, _P, C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "lg_render": (_I, [_P, C.POINTER(LgCamera), C.POINTER(LgRenderOpts), _P, _P, _P, C.POINTER(LgRenderStats)]),
    "lg_measure_read_bandwidth": (_I, [C.c_int, C.c_int, C.c_int64, C.c_int, C.POINTER(C.c_double)]),
    "lg_unet_wait_selftest": (_I, [_P, C.c_int64]),
    "lg_renderer_set_l2_window": (_I, [_P, C.c_int]),
    "lg_renderer_get_stack_bound": (_I, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "lg_renderer_set_top_records": (_I, [_P, C.c_int]),
    "lg_renderer_get_top_records": (_I, [_P]),
    "lg_render_sorted": (_I, [_P, C.POINTER(LgCamera), C.POINTER(LgRenderOpts), _P, _P, C.POINTER(LgRenderStats)]),
    "lg_render_device": (_I, [_P, C.POINTER(LgCamera), C.POINTER(LgRenderOpts), _P, C.POINTER(_P), C.POINTER(_P),
                              C.POINTER(_P)]),
    "lg_render_batch": (_I, [_P, C.POINTER(LgCamera), C.POINTER(LgRenderOpts), C.c_int32, _P, _P]),
    "lg_tonemap_device": (_I, [_P, _P, C.c_int64, C.c_float, _P]),
    "lg_render_gbuffer": (_I, [_P, C.POINTER(LgCamera), _P, _P, _P]),
    "lg_unet_create": (_I, [_I, _I, _I, C.POINTER(_P)]),
    "lg_unet_destroy": (None, [_P]),
    "lg_unet_num_params": (C.c_int64, [_P]),
    "lg_unet_set_params": (_I, [_P, _P, C.c_int64]),
    "lg_unet_get_params": (_I, [_P, _P, C.c_int64]),
    "lg_unet_forward": (_I, [_P, _P, _I, _I, _I, _P]),
    "lg_unet_forward_device": (_I, [_P, _P, _I, _I, _I, _P, _P]),
    "lg_unet_train_step": (_I, [_P, _P, _P, _I, _I, _I, C.c_float, C.POINTER(C.c_float)]),
    "lg_unet_train_step_async": (_I, [_P, _P, _P, _I, _I, _I, C.c_float, _P, _P]),
    "lg_unet_sync": (_I, [_P]),
    "lg_unet_loss_grad": (_I, [_P, _P, _P, _I, _I, _I, _P, C.POINTER(C.c_float)]),
    "lg_unet_adam_apply": (_I, [_P, C.c_float]),
    "lg_unet_adam_reset": (_I, [_P]),
    "lg_unet_autotune": (_I, [_P, _I, _I, _I, _I, _P]),
    "lg_unet_set_tiles": (_I, [_P, _P]),
    "lg_unet_set_fold_upsampling": (_I, [_P, _I]),
    "lg_conv3x3_device": (_I, [_P, _I, _I, _I, _I, _P, _I, _P, _I, C.c_float, _I, _P, _I, _I, _P, _I, _I, _P]),
    "lg_to_blocked_bf16": (_I, [_P, _I, _I, _I, _I, _P, _I, _P]),
    "lg_from_blocked_bf16": (_I, [_P, _I, _I, _I, _I, _P, _P]),
    "lg_rgb8_to_f32": (_I, [_P, _I, _I, _I, _P, _P]),
    "lg_f32_to_rgb8": (_I, [_P, _I, _I, _I, _P, _P]),
    "lg_accum_to_f32": (_I, [_P, _I, _I, _I, C.c_float, _P, _P]),
    "lg_f32_tonemap_rgb8": (_I, [_P, _I, _I, _I, _P, _P]),
    "lg_gather_crops": (_I, [_P, _I, _I, _I, _P, _P, _P, _I, _I, _P, _P]),
    "lg_write_png": (_I, [C.c_char_p, C.c_int32, C.c_int32, _P]),
    "lg_write_hdr": (_I, [C.c_char_p, C.c_int32, C.c_int32, _P]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads liblumina.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                               "(the CUDA library is required; there is no fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != LG_OK:
        raise LuminaError(rc, lib().lg_last_error().decode(errors="replace"))


def ptr(a) -> C.c_void_p:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "arrays passed to liblumina must be C-contiguous"
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a)
