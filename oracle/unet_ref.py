"""TEST INFRASTRUCTURE ONLY: the denoiser UNet in plain PyTorch (FP32/FP64).

Restates the reference network (LuminaGI-CudaRef ml/train.py:37-75) with the
same module names, so its state_dict keys and parameter order are the
reference's; pinned to the reference module by tests/golden/unet_golden.npz
(tests/golden/make_unet_golden.py).  Also provides:
  * make_params(seed): seeded He-normal initialisation, flat, state_dict order;
  * forward_bf16(model, x): the same network with BF16 rounding at exactly the
    points where this project's tensor-core kernels round (inputs and weights
    of every conv, every stored activation), FP32 everywhere else.
  * variant="hdr": the configuration-4 network the reference does not ship --
    ReLU, bilinear 2x upsampling (align_corners=False), log1p applied to the
    input and the residual taken in log space, output expm1(max(y, 0)).  Its
    loss (hdr_loss) is L1 between max(y, 0) and log1p(target).  Only this
    restatement defines it, so its parity is against this module alone.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn as nn
import torch.nn.functional as F


class ConvBlock(nn.Module):
    def __init__(self, cin, cout, slope=0.1):
        super().__init__()
        self.net = nn.Sequential(nn.Conv2d(cin, cout, 3, padding=1), nn.LeakyReLU(slope),
                                 nn.Conv2d(cout, cout, 3, padding=1), nn.LeakyReLU(slope))

    def forward(self, x):
        return self.net(x)


class UNetRef(nn.Module):
    """ml/train.py:51-75 (base 32; 3 or 12 input channels); variant "hdr" as above."""

    def __init__(self, base=32, in_ch=3, slope=0.1, variant="ref"):
        super().__init__()
        assert variant in ("ref", "hdr")
        self.variant = variant
        slope = 0.0 if variant == "hdr" else slope
        self.slope = slope
        self.d1 = ConvBlock(in_ch, base, slope)
        self.d2 = ConvBlock(base, base * 2, slope)
        self.d3 = ConvBlock(base * 2, base * 4, slope)
        self.d4 = ConvBlock(base * 4, base * 8, slope)
        self.u3 = ConvBlock(base * 8 + base * 4, base * 4, slope)
        self.u2 = ConvBlock(base * 4 + base * 2, base * 2, slope)
        self.u1 = ConvBlock(base * 2 + base, base, slope)
        self.tail = nn.Conv2d(base, 3, 1)

    def _up(self, t):
        if self.variant == "hdr":
            return F.interpolate(t, scale_factor=2, mode="bilinear", align_corners=False)
        return F.interpolate(t, scale_factor=2, mode="nearest")

    def forward_log(self, x):
        """hdr variant: max(log1p(x)[:, :3] + tail, 0) (the network output in log space)."""
        assert self.variant == "hdr"
        return torch.clamp(self._body(torch.log1p(x)), min=0.0)

    def _body(self, x):
        pool = lambda t: F.max_pool2d(t, 2)
        up = self._up
        d1 = self.d1(x)
        d2 = self.d2(pool(d1))
        d3 = self.d3(pool(d2))
        d4 = self.d4(pool(d3))
        u3 = self.u3(torch.cat([up(d4), d3], 1))
        u2 = self.u2(torch.cat([up(u3), d2], 1))
        u1 = self.u1(torch.cat([up(u2), d1], 1))
        return x[:, :3] + self.tail(u1)

    def forward(self, x):
        if self.variant == "hdr":
            return torch.expm1(self.forward_log(x))
        return torch.clamp(self._body(x), 0.0, 1.0)


def hdr_loss(model: UNetRef, x: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
    """Training loss of the hdr variant: L1 in log1p space."""
    return F.l1_loss(model.forward_log(x), torch.log1p(target))


def param_shapes(model: nn.Module):
    return [(k, tuple(v.shape)) for k, v in model.state_dict().items()]


def make_params(seed: int, model: nn.Module | None = None) -> np.ndarray:
    """He-normal conv weights (std sqrt(2/fan_in)), biases U(-0.05, 0.05); flat FP32, state_dict order."""
    model = model or UNetRef()
    rng = np.random.default_rng(seed)
    out = []
    for k, shp in param_shapes(model):
        if k.endswith("weight"):
            fan_in = int(np.prod(shp[1:]))
            out.append(rng.normal(0.0, np.sqrt(2.0 / fan_in), size=shp).astype(np.float32).ravel())
        else:
            out.append(rng.uniform(-0.05, 0.05, size=shp).astype(np.float32).ravel())
    return np.concatenate(out)


def load_flat(model: nn.Module, flat: np.ndarray) -> nn.Module:
    sd = model.state_dict()
    off = 0
    new = {}
    for k, v in sd.items():
        n = v.numel()
        new[k] = torch.from_numpy(np.asarray(flat[off:off + n], np.float32).reshape(v.shape).copy()).to(v.dtype)
        off += n
    assert off == len(flat), (off, len(flat))
    model.load_state_dict(new)
    return model


def flat_params(model: nn.Module) -> np.ndarray:
    return np.concatenate([v.detach().cpu().float().numpy().ravel() for v in model.state_dict().values()])


def forward_bf16(model: UNetRef, x: torch.Tensor, dtype=torch.float32, fold=(), log_out=False) -> torch.Tensor:
    """The network with BF16 rounding where the tensor-core kernels round;
    everything else in `dtype` (float64 gives the accumulation-order noise
    floor of the FP32 version).

    fold: names of the decoder blocks ("u3", "u2", "u1") whose first conv runs
    the library's folded-upsampling form.  Nearest upsampling repeats each
    row, so an even output row 2r reads low-resolution rows r-1 (tap ky0) and
    r (ky1 + ky2), an odd row 2r+1 rows r (ky0 + ky1) and r+1 (ky2); the
    library sums those taps of the upsampled channels in FP32 and rounds the
    sum to BF16 once.  Here: the conv over the upsampled input with those
    rounded weights, even output rows from one weight set and odd rows from
    the other (exact, since rows 2r and 2r+1 of the input are equal).

    log_out: for the hdr variant, return the log-space output max(log1p(x) +
    tail, 0) that hdr_loss compares with log1p(target), not its expm1."""
    s = model.slope

    def _q(t):
        return t.to(torch.bfloat16).to(dtype)

    x = x.to(dtype)
    hdr = getattr(model, "variant", "ref") == "hdr"
    if hdr:
        x = torch.log1p(x)

    def conv(block_conv, t):
        return F.conv2d(_q(t), _q(block_conv.weight.to(dtype)), block_conv.bias.to(dtype), padding=1)

    def conv_folded(block_conv, t, up_c):
        w = block_conv.weight.to(dtype)
        u = w[:, :up_c]
        we, wo = _q(w), _q(w)
        we[:, :up_c, 0], we[:, :up_c, 1], we[:, :up_c, 2] = _q(u[:, :, 0]), _q(u[:, :, 1] + u[:, :, 2]), 0.0
        wo[:, :up_c, 0], wo[:, :up_c, 1], wo[:, :up_c, 2] = _q(u[:, :, 0] + u[:, :, 1]), 0.0, _q(u[:, :, 2])
        b = block_conv.bias.to(dtype)
        y = F.conv2d(_q(t), we, b, padding=1)
        y[:, :, 1::2] = F.conv2d(_q(t), wo, b, padding=1)[:, :, 1::2]
        return y

    def block(b, t, name=None, up_c=0):
        first = conv_folded(b.net[0], t, up_c) if name in fold else conv(b.net[0], t)
        t = _q(F.leaky_relu(first, s))
        return _q(F.leaky_relu(conv(b.net[2], t), s))

    pool = lambda t: F.max_pool2d(t, 2)
    if hdr:  # interpolated from the stored (BF16) low-resolution output, stored again as BF16
        up = lambda t: _q(F.interpolate(t, scale_factor=2, mode="bilinear", align_corners=False))
    else:
        up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")
    d1 = block(model.d1, x)
    d2 = block(model.d2, pool(d1))
    d3 = block(model.d3, pool(d2))
    d4 = block(model.d4, pool(d3))
    if hdr:
        fold = ()  # bilinear upsampling does not repeat rows
    u3 = block(model.u3, torch.cat([up(d4), d3], 1), "u3", d4.shape[1])
    u2 = block(model.u2, torch.cat([up(u3), d2], 1), "u2", u3.shape[1])
    u1 = block(model.u1, torch.cat([up(u2), d1], 1), "u1", u2.shape[1])
    tail = F.conv2d(u1, model.tail.weight.to(dtype), model.tail.bias.to(dtype))
    if hdr:
        y = torch.clamp(x[:, :3] + tail, min=0.0)
        return y if log_out else torch.expm1(y)
    return torch.clamp(x[:, :3] + tail, 0.0, 1.0)
