"""The learned surrogate end to end: the UNet standing in for extra samples.

  1. On-device data: P camera poses on the seeded orbit of the engine-scale
     scene, each rendered at a noisy and a clean sample count (the pairs the
     reference produced with ml/gen_dataset.py + cuda_ref --batch, here
     rendered straight into device buffers and converted u8/255 as
     ml/train.py reads its PNGs).
  2. Training (ml/train.py:128-225 semantics): per epoch, `crops_per_image`
     random square crops of every training pose, shuffled into batches
     (the last one partial); L1 loss; Adam; validation L1 on crops of the
     held-out poses; the best-validation parameters are kept and saved in the
     reference checkpoint format {"model", "base", "in_ch"}.
     With --variant hdr the network is the configuration-4 one (ReLU,
     bilinear upsampling, log1p HDR radiance in/out) trained on accum/spp.
     With --gbuffer the network is train.py's 12-channel variant: the input
     stacks the noisy colour with the albedo, normal and position images of
     the G-buffer pass (train.py:112-119); the residual stays on colour.
  3. Evaluation on held-out poses against a judge rendered with FP64
     per-pixel accumulators: PSNR / SSIM of the 8-bit sqrt-tonemapped images
     (tools/diff.py) for the noisy render, the denoised render and the plain
     clean render, and the device time of each path.

Run:  python -m lumina.surrogate --out results.json [options]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time

import numpy as np

from . import _ffi, metrics
from .render import Renderer
from .scene import ENGINE_CENTER, engine_scene, orbit_poses
from .unet import UNet, unflatten


def _torch():
    import torch
    return torch


def render_to_f32(r: Renderer, cam, spp: int, bounces: int, out_ptr: int, sample_base: int = 0, hdr: bool = False):
    """Renders one frame into 3 x H x W FP32 at out_ptr: its tonemapped u8/255
    image (reference variant) or its linear radiance accum/spp (hdr)."""
    c = cam.to_c()
    o = _ffi.LgRenderOpts(spp, bounces, sample_base, 0)
    rgb, acc = C.c_void_p(), C.c_void_p()
    _ffi.check(_ffi.lib().lg_render_device(r._h, C.byref(c), C.byref(o), None, C.byref(rgb), C.byref(acc), None))
    H, W = int(cam.height), int(cam.width)
    if hdr:
        _ffi.check(_ffi.lib().lg_accum_to_f32(acc, 1, H, W, 1.0 / spp, C.c_void_p(out_ptr), None))
    else:
        _ffi.check(_ffi.lib().lg_rgb8_to_f32(rgb, 1, H, W, C.c_void_p(out_ptr), None))


def judge_u8(r: Renderer, cam, spp: int, bounces: int) -> np.ndarray:
    """High-spp judge image from FP64 accumulators, tonemapped as the renderer does."""
    out = r.render(camera=cam, spp=spp, bounces=bounces, accum=False, accum64=True, rgb=False)
    lin = (out["accum64"] / spp).astype(np.float32)
    return metrics.tonemap_u8(lin)


def gbuffer_to_f32(r: Renderer, cam, out_ptr: int) -> None:
    """G-buffer pass (albedo, normal, position; u8/255) into 9 FP32 planes at out_ptr."""
    torch = _torch()
    H, W = int(cam.height), int(cam.width)
    planes = torch.from_numpy(np.stack(r.gbuffer(cam))).cuda()  # (3, H, W, 3) u8
    _ffi.check(_ffi.lib().lg_rgb8_to_f32(C.c_void_p(planes.data_ptr()), 3, H, W, C.c_void_p(out_ptr), None))
    torch.cuda.synchronize()


def make_input(r: Renderer, cam, spp: int, bounces: int, out, sample_base: int = 0, hdr: bool = False) -> None:
    """Network input of one frame into out (C x H x W, C = 3 or 12): the
    render, then for 12 channels the G-buffer images after it."""
    render_to_f32(r, cam, spp, bounces, out.data_ptr(), sample_base, hdr)
    if out.shape[0] == 12:
        gbuffer_to_f32(r, cam, out[3].data_ptr())


def make_dataset(r: Renderer, cams, noisy_spp: int, clean_spp: int, bounces: int, in_ch: int = 3,
                 hdr: bool = False):
    torch = _torch()
    H, W = int(cams[0].height), int(cams[0].width)
    noisy = torch.empty((len(cams), in_ch, H, W), device="cuda")
    clean = torch.empty((len(cams), 3, H, W), device="cuda")
    for i, cam in enumerate(cams):
        make_input(r, cam, noisy_spp, bounces, noisy[i], hdr=hdr)
        # a disjoint sample range keeps the clean target independent of the noisy input
        render_to_f32(r, cam, clean_spp, bounces, clean[i].data_ptr(), sample_base=100000, hdr=hdr)
    torch.cuda.synchronize()
    return noisy, clean


def gather(images, idx, ys, xs, crop, out=None, stream: int = 0):
    """Crops (all channels) of FP32 NCHW images; C a multiple of 3: a C-channel
    image is gathered as C/3 consecutive 3-channel images.  With a stream
    handle the copy is only queued there."""
    torch = _torch()
    n = len(idx)
    I, Cc, Hh, Ww = images.shape
    g = Cc // 3
    if out is None:
        out = torch.empty((n, Cc, crop, crop), device="cuda")
    a = lambda v: np.ascontiguousarray(v, np.int32)
    ii = a((np.asarray(idx, np.int64)[:, None] * g + np.arange(g)[None, :]).reshape(-1))
    yy, xx = a(np.repeat(ys, g)), a(np.repeat(xs, g))
    _ffi.check(_ffi.lib().lg_gather_crops(C.c_void_p(images.data_ptr()), I * g, Hh, Ww, _ffi.ptr(ii), _ffi.ptr(yy),
                                          _ffi.ptr(xx), n * g, crop, C.c_void_p(out.data_ptr()),
                                          C.c_void_p(stream) if stream else None))
    return out


def train(net: UNet, noisy, clean, train_idx, val_idx, epochs=120, batch=16, crop=128, lr=1e-4, crops_per_image=1,
          seed=42, log=print):
    """ml/train.py:184-217: returns (best params, history).

    The batches of an epoch are queued without waiting for the GPU: crops are
    gathered into one pair of buffers on a stream of this loop, and each
    step (lg_unet_train_step_async) is ordered on that stream, so the next
    gather waits for the step that reads the buffers.  The training loss is
    summed on the device and read once per epoch; validation (synchronous)
    follows, as in the reference loop."""
    torch = _torch()
    rng = np.random.RandomState(seed)
    H, W = noisy.shape[2], noisy.shape[3]
    best, best_val, hist = None, float("inf"), []
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        xbuf = torch.empty((batch, noisy.shape[1], crop, crop), device="cuda")
        tbuf = torch.empty((batch, clean.shape[1], crop, crop), device="cuda")
        loss_sum = torch.zeros(1, device="cuda")
    for ep in range(epochs):
        order = np.repeat(np.asarray(train_idx), crops_per_image)
        rng.shuffle(order)
        ys = rng.randint(0, H - crop + 1, len(order))
        xs = rng.randint(0, W - crop + 1, len(order))
        seen = 0
        with torch.cuda.stream(stream):
            loss_sum.zero_()
            for b0 in range(0, len(order), batch):
                sl = slice(b0, b0 + batch)
                n = len(order[sl])
                xb = gather(noisy, order[sl], ys[sl], xs[sl], crop, xbuf[:n], sh)
                tb = gather(clean, order[sl], ys[sl], xs[sl], crop, tbuf[:n], sh)
                net.train_step_async(xb.data_ptr(), tb.data_ptr(), n, crop, crop, lr, loss_sum.data_ptr(), sh)
                seen += n
            tl = float(loss_sum.item())
        net.sync()
        vy = rng.randint(0, H - crop + 1, len(val_idx))
        vx = rng.randint(0, W - crop + 1, len(val_idx))
        xv = gather(noisy, val_idx, vy, vx, crop)
        tv = gather(clean, val_idx, vy, vx, crop)
        vl, _ = net.loss_grad(xv.data_ptr(), tv.data_ptr(), len(val_idx), crop, crop)
        tag = ""
        if vl < best_val:
            best_val, best, tag = vl, net.get_params(), "  *"
        hist.append((ep + 1, tl / seen, vl))
        if log and ((ep + 1) % max(1, epochs // 12) == 0 or ep == 0):
            log(f"epoch {ep + 1:3d}/{epochs}  train={tl / seen:.4f}  val={vl:.4f}{tag}")
    return best, best_val, hist


def save_checkpoint(params: np.ndarray, path: str, in_ch: int = 3, variant: str = "ref") -> None:
    """Reference checkpoint format (ml/train.py:216), loadable by tools/denoise.py;
    the hdr variant adds "variant": "hdr"."""
    torch = _torch()
    sd = {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in unflatten(params, in_ch).items()}
    ck = {"model": sd, "base": 32, "in_ch": in_ch}
    if variant != "ref":
        ck["variant"] = variant
    torch.save(ck, path)


def eval_frames(r: Renderer, cams, noisy_spp, clean_spp, judge_spp, bounces, in_ch: int = 3, hdr: bool = False):
    """Held-out frames: judge (FP64 accumulators), noisy and clean renders with their device times."""
    torch = _torch()
    H, W = int(cams[0].height), int(cams[0].width)
    assert H % 8 == 0 and W % 8 == 0, "evaluation frames must be multiples of 8"
    out = []
    for cam in cams:
        judge = judge_u8(r, cam, judge_spp, bounces)
        noisy = r.render(camera=cam, spp=noisy_spp, bounces=bounces, accum=False)
        clean = r.render(camera=cam, spp=clean_spp, bounces=bounces, accum=False, sample_base=100000)
        x = torch.empty((1, in_ch, H, W), device="cuda")
        make_input(r, cam, noisy_spp, bounces, x[0], hdr=hdr)
        out.append({"judge": judge, "noisy": noisy["rgb"], "clean": clean["rgb"], "x": x,
                    "noisy_ms": noisy["kernel_ms"], "clean_ms": clean["kernel_ms"]})
    return out


def evaluate(net: UNet, frames):
    """PSNR/SSIM of noisy, denoised and clean renders vs the judge; device times."""
    torch = _torch()
    rows = []
    for f in frames:
        x = f["x"]
        _, _, H, W = x.shape
        y = torch.empty((1, 3, H, W), device="cuda")
        u8 = torch.empty((H * W * 3,), dtype=torch.uint8, device="cuda")
        st = torch.cuda.current_stream()
        net.forward_device(x.data_ptr(), 1, H, W, y.data_ptr(), st.cuda_stream)  # warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        net.forward_device(x.data_ptr(), 1, H, W, y.data_ptr(), st.cuda_stream)
        e1.record(st)
        to_u8 = _ffi.lib().lg_f32_tonemap_rgb8 if net.variant == "hdr" else _ffi.lib().lg_f32_to_rgb8
        _ffi.check(to_u8(C.c_void_p(y.data_ptr()), 1, H, W, C.c_void_p(u8.data_ptr()), C.c_void_p(st.cuda_stream)))
        torch.cuda.synchronize()
        den = u8.cpu().numpy().reshape(H, W, 3)
        row = {"noisy_ms": f["noisy_ms"], "unet_ms": e0.elapsed_time(e1), "clean_ms": f["clean_ms"]}
        for name, img in (("noisy", f["noisy"]), ("denoised", den), ("clean", f["clean"])):
            row[f"{name}_psnr"] = metrics.psnr(img, f["judge"])
            row[f"{name}_ssim"] = metrics.ssim(img, f["judge"])
        rows.append(row)
    agg = {k: float(np.mean([r_[k] for r_ in rows])) for k in rows[0]}
    agg["speedup_clean_over_denoised"] = agg["clean_ms"] / (agg["noisy_ms"] + agg["unet_ms"])
    agg["gap_db_clean_minus_denoised"] = agg["clean_psnr"] - agg["denoised_psnr"]
    return agg, rows


def he_init(seed: int, in_ch: int = 3) -> np.ndarray:
    """Seeded He-normal conv weights, zero biases, state_dict order."""
    from .unet import param_shapes
    rng = np.random.default_rng(seed)
    out = []
    for k, shp in param_shapes(in_ch):
        if k.endswith("weight"):
            fan_in = int(np.prod(shp[1:]))
            out.append(rng.normal(0, math.sqrt(2.0 / fan_in), shp).astype(np.float32).ravel())
        else:
            out.append(np.zeros(shp, np.float32).ravel())
    return np.concatenate(out)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="surrogate_results.json")
    ap.add_argument("--poses", type=int, default=50)
    ap.add_argument("--val", type=int, default=5)
    ap.add_argument("--noisy-spp", type=int, default=8)
    ap.add_argument("--clean-spp", type=int, default=256)
    ap.add_argument("--judge-spp", type=int, default=1024)
    ap.add_argument("--bounces", type=int, default=2)
    ap.add_argument("--recipe", action="append", default=[],
                    help="name:epochs:batch:crop:lr:crops_per_image (repeatable); "
                         "default: the 120-epoch config recipe")
    ap.add_argument("--width", type=int, default=1728)
    ap.add_argument("--height", type=int, default=864)
    ap.add_argument("--checkpoint", default="")
    ap.add_argument("--save-npz", default="",
                    help="also write the best parameters of each recipe as <path>.<recipe>.npz (FP16, state_dict "
                         "order, with the held-out pose indices)")
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--gbuffer", action="store_true", help="12-channel network on colour + G-buffer (train.py --gbuffer)")
    ap.add_argument("--variant", default="ref", choices=["ref", "hdr"],
                    help="ref: the reference network on u8/255 frames; hdr: ReLU, bilinear, log1p HDR radiance")
    a = ap.parse_args(argv)
    in_ch = 12 if a.gbuffer else 3
    hdr = a.variant == "hdr"
    torch = _torch()
    t0 = time.time()
    sc = engine_scene(seed=7, width=a.width, height=a.height)
    r = Renderer(0)
    r.set_scene(sc)
    cams = [sc.camera.look_at(p, t) for p, t in orbit_poses(a.poses, seed=11, center=ENGINE_CENTER)]
    noisy, clean = make_dataset(r, cams, a.noisy_spp, a.clean_spp, a.bounces, in_ch, hdr)
    t_data = time.time() - t0
    perm = np.random.RandomState(a.seed).permutation(a.poses)
    val_idx, train_idx = perm[:a.val].tolist(), perm[a.val:].tolist()
    t1 = time.time()
    frames = eval_frames(r, [cams[i] for i in val_idx], a.noisy_spp, a.clean_spp, a.judge_spp, a.bounces, in_ch, hdr)
    t_judge = time.time() - t1
    recipes = a.recipe or ["config:120:16:128:1e-4:1"]
    res = {"config": vars(a), "triangles": sc.n_tris, "train_poses": len(train_idx), "val_poses": len(val_idx),
           "data_seconds": t_data, "eval_render_seconds": t_judge, "recipes": {}}
    for spec in recipes:
        name, ep, bs, cr, lr, cpi = spec.split(":")
        net = UNet(in_ch=in_ch, variant=a.variant)
        net.set_params(he_init(a.seed, in_ch))
        t2 = time.time()
        best, best_val, hist = train(net, noisy, clean, train_idx, val_idx, int(ep), int(bs), int(cr), float(lr),
                                     int(cpi), a.seed, log=lambda m: print(f"[{name}] {m}", flush=True))
        t_train = time.time() - t2
        net.set_params(best)
        if a.checkpoint:
            save_checkpoint(best, f"{a.checkpoint}.{name}.pt", in_ch, a.variant)
        if a.save_npz:
            np.savez_compressed(f"{a.save_npz}.{name}.npz", params=best.astype(np.float16),
                                val_idx=np.asarray(val_idx, np.int32), poses=np.int32(a.poses), in_ch=np.int32(in_ch),
                                variant=np.bytes_(a.variant), recipe=np.bytes_(spec))
        agg, rows = evaluate(net, frames)
        res["recipes"][name] = {"spec": spec, "train_seconds": t_train, "best_val_l1": best_val,
                                "history_tail": hist[-3:], "eval": agg, "per_pose": rows}
        print(json.dumps({"recipe": name, "eval": agg, "best_val_l1": best_val, "train_seconds": t_train}),
              flush=True)
        net.close()
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    r.close()


if __name__ == "__main__":
    main()
