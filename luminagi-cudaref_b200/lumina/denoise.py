"""denoise -- drop-in for the reference's tools/denoise.py on the tensor-core UNet.

    python -m lumina.denoise <checkpoint.pt> <noisy.png> <out.png>
                             [--albedo A.png --normal N.png --worldpos P.png]

Loads a reference-format checkpoint {"model", "base", "in_ch"} (ml/train.py:216),
reads the PNG as u8/255, replicate-pads to multiples of 8, runs the network,
crops, writes (clip*255 + 0.5) as u8 (tools/denoise.py:34-52) and prints
"inference: <ms> ms (<W>x<H>, base=<b>)  wrote <out>" with the device time of
the forward pass.  A 12-channel (--gbuffer) checkpoint, which the reference
script rejects, also takes the G-buffer images; by default they are the
<stem>.albedo.png, <stem>.normal.png and <stem>.worldpos.png files that
`cuda_ref --gbuffer` writes beside <noisy.png>.
"""
from __future__ import annotations

import argparse
import pathlib
import sys
import time

import numpy as np

from ._ffi import check, lib
from .image import load_image
from .unet import UNet


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("checkpoint")
    ap.add_argument("noisy_png")
    ap.add_argument("out_png")
    ap.add_argument("--albedo")
    ap.add_argument("--normal")
    ap.add_argument("--worldpos")
    a = ap.parse_args(argv)

    import torch
    ck = torch.load(a.checkpoint, map_location="cpu", weights_only=True)
    base, in_ch = ck.get("base", 32), ck.get("in_ch", 3)
    if in_ch not in (3, 12):
        sys.exit(f"checkpoint expects {in_ch}-ch input; not supported by this script")
    if ck.get("variant", "ref") != "ref":
        sys.exit("checkpoint is the HDR variant (radiance in/out); this script denoises 8-bit PNGs")
    net = UNet(base=base, in_ch=in_ch)
    net.load_state_dict(ck["model"])

    img = load_image(a.noisy_png)[..., :3]
    planes = [img]
    if in_ch == 12:
        stem = pathlib.Path(a.noisy_png).with_suffix("")
        for name in ("albedo", "normal", "worldpos"):
            p = getattr(a, name) or f"{stem}.{name}.png"
            planes.append(load_image(p)[..., :3])
    H, W = img.shape[:2]
    x = np.concatenate([p.astype(np.float32) / 255.0 for p in planes], axis=2)
    ph, pw = (8 - H % 8) % 8, (8 - W % 8) % 8
    x = np.pad(x, ((0, ph), (0, pw), (0, 0)), mode="edge").transpose(2, 0, 1)[None]
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dy = torch.empty((1, 3, H + ph, W + pw), device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    net.forward_device(dx.data_ptr(), 1, H + ph, W + pw, dy.data_ptr())
    torch.cuda.synchronize()
    dt_ms = (time.perf_counter() - t0) * 1000.0
    y = dy[0, :, :H, :W].cpu().numpy().transpose(1, 2, 0)
    out = np.ascontiguousarray((np.clip(y, 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8))
    check(lib().lg_write_png(str(a.out_png).encode(), W, H, out.ctypes.data))
    print(f"inference: {dt_ms:.1f} ms ({W}x{H}, base={base})  wrote {a.out_png}")
    net.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
