"""lumina -- B200 render path of LuminaGI-CudaRef behind a C ABI.

scene.json -> device LBVH -> path trace -> tonemap -> PNG, driven from Python
through ctypes (lumina._ffi).  All work runs in liblumina.so's CUDA kernels.
"""
from ._ffi import LIB_PATH, CLI_PATH, LuminaError, lib  # noqa: F401
from .scene import Camera, Scene, box_scene, engine_scene, orbit_poses, look_at_camera  # noqa: F401
from .render import Renderer, build_bvh  # noqa: F401
from .unet import UNet  # noqa: F401,E402
from .image import load_image  # noqa: F401,E402
