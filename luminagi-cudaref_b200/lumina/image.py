"""PNG decoding through liblumina (stbi_load(..., 4) semantics for PNG files)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._ffi import LG_ERR_IO, LuminaError, lib


def load_image(path: str) -> np.ndarray:
    """Decodes a PNG file to (H, W, 4) uint8 RGBA.  Raises OSError when the
    file cannot be read or is not a supported PNG."""
    w, h = C.c_int32(), C.c_int32()
    px = C.POINTER(C.c_uint8)()
    rc = lib().lg_image_load(str(path).encode(), C.byref(w), C.byref(h), C.byref(px))
    if rc != 0:
        msg = lib().lg_last_error().decode(errors="replace")
        if rc == LG_ERR_IO:
            raise FileNotFoundError(msg)
        raise OSError(str(LuminaError(rc, msg)))
    try:
        return np.ctypeslib.as_array(px, shape=(h.value, w.value, 4)).copy()
    finally:
        lib().lg_image_free(px)
