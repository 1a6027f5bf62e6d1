"""The denoiser (reference ml/train.py UNet) on liblumina's tensor-core kernels.

`UNet` holds FP32 master parameters in the reference's state_dict order and
runs the BF16 tcgen05 forward pass.  `denoise_rgb8` follows tools/denoise.py:
u8/255, replicate-pad to multiples of 8, run, crop, clip*255+0.5.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._ffi import LG_UNET_HDR_VARIANT, LG_UNET_RELU, check, lib, ptr

# state_dict keys and shapes of the reference UNet(base=32, in_ch).
_BLOCKS = [("d1", None, 32), ("d2", 32, 64), ("d3", 64, 128), ("d4", 128, 256), ("u3", 384, 128), ("u2", 192, 64),
           ("u1", 96, 32)]


def param_shapes(in_ch: int = 3):
    out = []
    for name, cin, cout in _BLOCKS:
        cin = in_ch if cin is None else cin
        out += [(f"{name}.net.0.weight", (cout, cin, 3, 3)), (f"{name}.net.0.bias", (cout,)),
                (f"{name}.net.2.weight", (cout, cout, 3, 3)), (f"{name}.net.2.bias", (cout,))]
    return out + [("tail.weight", (3, 32, 1, 1)), ("tail.bias", (3,))]


PARAM_SHAPES = param_shapes(3)
N_PARAMS = int(sum(np.prod(s) for _, s in PARAM_SHAPES))


def flatten_state_dict(sd, in_ch: int = 3) -> np.ndarray:
    """Reference state_dict (tensors or arrays) -> flat FP32 in key order."""
    out = []
    for k, shp in param_shapes(in_ch):
        v = sd[k]
        v = v.detach().cpu().float().numpy() if hasattr(v, "detach") else np.asarray(v, np.float32)
        assert tuple(v.shape) == shp, (k, v.shape, shp)
        out.append(v.ravel())
    return np.concatenate(out).astype(np.float32)


def unflatten(flat: np.ndarray, in_ch: int = 3) -> dict:
    out, off = {}, 0
    for k, shp in param_shapes(in_ch):
        n = int(np.prod(shp))
        out[k] = flat[off:off + n].reshape(shp)
        off += n
    return out


class UNet:
    """variant "ref": the reference network (LeakyReLU 0.1, nearest upsampling,
    [0,1] images, clamped residual); "hdr": ReLU, bilinear upsampling, HDR
    radiance in and out through log1p/expm1 (the configuration-4 network).
    act="relu" swaps only the activation of the reference variant."""

    def __init__(self, base: int = 32, in_ch: int = 3, act: str = "leaky", variant: str = "ref"):
        self._h = C.c_void_p()
        assert variant in ("ref", "hdr")
        mode = LG_UNET_HDR_VARIANT if variant == "hdr" else (0 if act == "leaky" else LG_UNET_RELU)
        check(lib().lg_unet_create(base, in_ch, mode, C.byref(self._h)))
        self.in_ch = in_ch
        self.variant = variant
        self.n_params = int(lib().lg_unet_num_params(self._h))
        assert self.n_params == int(sum(np.prod(s) for _, s in param_shapes(in_ch)))

    def close(self):
        if self._h:
            lib().lg_unet_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, flat: np.ndarray) -> None:
        flat = np.ascontiguousarray(flat, np.float32)
        check(lib().lg_unet_set_params(self._h, ptr(flat), len(flat)))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        check(lib().lg_unet_get_params(self._h, ptr(out), len(out)))
        return out

    def load_state_dict(self, sd) -> None:
        self.set_params(flatten_state_dict(sd, self.in_ch))

    def load_checkpoint(self, path: str) -> None:
        """Loads a reference checkpoint dict {"model": state_dict, "base", "in_ch"} (ml/train.py:216)."""
        import torch
        ck = torch.load(path, map_location="cpu", weights_only=True)
        if ck.get("base", 32) != 32 or ck.get("in_ch", 3) != self.in_ch or ck.get("variant", "ref") != self.variant:
            raise ValueError(f"checkpoint is base={ck.get('base', 32)}, in_ch={ck.get('in_ch', 3)}, "
                             f"variant={ck.get('variant', 'ref')}; this UNet is base=32, in_ch={self.in_ch}, "
                             f"variant={self.variant}")
        self.load_state_dict(ck["model"])

    def forward(self, x: np.ndarray) -> np.ndarray:
        """x: (N,in_ch,H,W) FP32 in [0,1], H and W multiples of 8; returns (N,3,H,W)."""
        x = np.ascontiguousarray(x, np.float32)
        n, c, h, w = x.shape
        assert c == self.in_ch
        y = np.empty((n, 3, h, w), np.float32)
        check(lib().lg_unet_forward(self._h, ptr(x), n, h, w, ptr(y)))
        return y

    def forward_device(self, d_x: int, n: int, h: int, w: int, d_y: int, stream: int = 0) -> None:
        check(lib().lg_unet_forward_device(self._h, C.c_void_p(d_x), n, h, w, C.c_void_p(d_y),
                                           C.c_void_p(stream) if stream else None))

    def train_step(self, d_x: int, d_target: int, n: int, h: int, w: int, lr: float) -> float:
        """One L1 + Adam step on device FP32 NCHW batches; returns the loss before the update."""
        loss = C.c_float(0)
        check(lib().lg_unet_train_step(self._h, C.c_void_p(d_x), C.c_void_p(d_target), n, h, w, lr, C.byref(loss)))
        return float(loss.value)

    def train_step_async(self, d_x: int, d_target: int, n: int, h: int, w: int, lr: float, d_loss_sum: int = 0,
                         stream: int = 0) -> None:
        """The same step queued on `stream` (a CUDA stream handle) without waiting for the device; n x the
        batch's mean loss is added to the device float at d_loss_sum (0: none).  See sync()."""
        check(lib().lg_unet_train_step_async(self._h, C.c_void_p(d_x), C.c_void_p(d_target), n, h, w, lr,
                                             C.c_void_p(d_loss_sum) if d_loss_sum else None,
                                             C.c_void_p(stream) if stream else None))

    def sync(self) -> None:
        """Waits for the queued steps; raises if a tensor-core kernel gave up a wait."""
        check(lib().lg_unet_sync(self._h))

    def loss_grad(self, d_x: int, d_target: int, n: int, h: int, w: int):
        """(loss, flat FP32 gradient) without updating the parameters."""
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_float(0)
        check(lib().lg_unet_loss_grad(self._h, C.c_void_p(d_x), C.c_void_p(d_target), n, h, w, ptr(g), C.byref(loss)))
        return float(loss.value), g

    def adam_apply(self, lr: float) -> None:
        """Adam step with the gradients of the last loss_grad call."""
        check(lib().lg_unet_adam_apply(self._h, lr))

    def adam_reset(self) -> None:
        check(lib().lg_unet_adam_reset(self._h))

    def autotune(self, n: int, h: int, w: int, backward: bool = False):
        """Times every compiled conv tile shape and kernel per layer at n x h x w and
        keeps the fastest (lg_unet_autotune); returns 30 (bn, kc, stages, kernel) quadruples, kernel 0..7 as
        include/lumina.h lists them."""
        out = np.zeros(120, np.int32)
        check(lib().lg_unet_autotune(self._h, n, h, w, 1 if backward else 0, ptr(out)))
        return [tuple(int(v) for v in out[4 * i:4 * i + 4]) for i in range(30)]

    def set_tiles(self, tiles) -> None:
        """30 (bn, kc, stages, kernel) choices as autotune returns them; (0, 0, 0, 0) = default."""
        arr = np.ascontiguousarray(np.asarray(tiles, np.int32).reshape(120))
        check(lib().lg_unet_set_tiles(self._h, ptr(arr)))

    def set_fold_upsampling(self, on: bool) -> None:
        """Inference passes of u3a, u2a, u1a on the x-only upsampled lower level with row taps summed per
        output-row parity (lg_unet_set_fold_upsampling; on by default, nearest upsampling only)."""
        check(lib().lg_unet_set_fold_upsampling(self._h, 1 if on else 0))

    def denoise_hdr(self, radiance: np.ndarray) -> np.ndarray:
        """HDR variant: (H,W,3) FP32 linear radiance -> (H,W,3), edge-padded to multiples of 8."""
        assert self.variant == "hdr" and self.in_ch == 3
        H, W = radiance.shape[:2]
        ph, pw = (8 - H % 8) % 8, (8 - W % 8) % 8
        x = np.pad(np.asarray(radiance, np.float32), ((0, ph), (0, pw), (0, 0)), mode="edge")
        return self.forward(x.transpose(2, 0, 1)[None])[0].transpose(1, 2, 0)[:H, :W].copy()

    def denoise_rgb8(self, img: np.ndarray, albedo=None, normal=None, worldpos=None) -> np.ndarray:
        """tools/denoise.py:34-52: (H,W,3) u8 -> (H,W,3) u8.  A 12-channel
        network also takes the G-buffer images (H,W,3) u8, stacked after the
        colour as the reference's --gbuffer dataset stacks them (train.py:112-119)."""
        planes = [img] + ([albedo, normal, worldpos] if self.in_ch == 12 else [])
        assert all(p is not None for p in planes), "a 12-channel network needs albedo, normal and worldpos"
        x = np.concatenate([p.astype(np.float32) / 255.0 for p in planes], axis=2)
        H, W = x.shape[:2]
        ph, pw = (8 - H % 8) % 8, (8 - W % 8) % 8
        x = np.pad(x, ((0, ph), (0, pw), (0, 0)), mode="edge")
        y = self.forward(x.transpose(2, 0, 1)[None])[0].transpose(1, 2, 0)[:H, :W]
        return (np.clip(y, 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)
