"""Device-timed micro-benchmarks of the library's kernels.

    python -m lumina.perf unet  [--n 1] [--h 864] [--w 1728] [--reps 10] [--kernel default|single|autotune] [--fold 1|0]
    python -m lumina.perf trace [--spp 8] [--bounces 2] [--width 4] [--reps 2]
    python -m lumina.perf bvh   [--reps 5]
    python -m lumina.perf batch [--poses 50] [--spp 8] [--bounces 2]
    python -m lumina.perf membench

Prints one JSON line.  Used for the profiles (run under ncu) and for quick
A/B measurements; bench.py is the benchmark of record.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


# Forward convs (d1a .. u1b) on the persistent kernel with resident weights
# where the layer has one output block and its weights fit beside the ring.
RESIDENT_TILES = [(32, 16, 10, 2), (32, 32, 6, 2), (64, 32, 4, 2), (64, 32, 4, 2)] + [(0, 0, 0, 1)] * 7 + \
                 [(64, 32, 4, 2), (32, 32, 5, 2), (32, 32, 6, 2)]
# The same layers with resident weights on 4-row tiles.
ROWS4_TILES = [(32, 16, 8, 3), (32, 32, 4, 3), (64, 32, 3, 3), (64, 32, 3, 3)] + [(0, 0, 0, 1)] * 7 + \
              [(64, 32, 3, 3), (32, 32, 3, 3), (32, 32, 4, 3)]
# Every layer with 32 or 64 output channels with the row taps packed into N:
# 4-row tiles (choice 4 resident weights, 6 streamed for u2a) ...
DYP4_TILES = [(32, 16, 7, 4), (32, 32, 3, 4), (64, 32, 3, 4), (64, 32, 2, 4)] + [(0, 0, 0, 1)] * 6 + \
             [(64, 32, 2, 6), (64, 32, 2, 4), (32, 32, 3, 4), (32, 32, 3, 4)]
# ... and 8-row tiles for the 32-channel layers (5 resident, 7 streamed for u1a).
DYP8_TILES = [(32, 16, 4, 5), (32, 32, 2, 5), (64, 32, 3, 4), (64, 32, 2, 4)] + [(0, 0, 0, 1)] * 6 + \
             [(64, 32, 2, 6), (64, 32, 2, 4), (32, 32, 2, 7), (32, 32, 2, 5)]

def unet(a):
    import torch

    from .unet import UNet
    net = UNet(variant=a.variant)
    net.set_params(np.random.default_rng(5).normal(0, 0.02, net.n_params).astype(np.float32))
    tiles = None
    if a.kernel == "single":
        net.set_tiles([(0, 0, 0, 0)] * 30)
    elif a.kernel == "resident":
        net.set_tiles(RESIDENT_TILES + [(0, 0, 0, 1)] * 16)
    elif a.kernel == "rows4":
        net.set_tiles(ROWS4_TILES + [(0, 0, 0, 1)] * 16)
    elif a.kernel == "dyp4":
        net.set_tiles(DYP4_TILES + [(0, 0, 0, 1)] * 16)
    elif a.kernel == "dyp8":
        net.set_tiles(DYP8_TILES + [(0, 0, 0, 1)] * 16)
    net.set_fold_upsampling(bool(a.fold))
    if a.kernel == "autotune":
        tiles = net.autotune(a.n, a.h, a.w)[:14]
    x = torch.rand((a.n, 3, a.h, a.w), device="cuda")
    y = torch.empty_like(x)
    st = torch.cuda.current_stream()
    for _ in range(3):
        net.forward_device(x.data_ptr(), a.n, a.h, a.w, y.data_ptr(), st.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    e0.record(st)
    for _ in range(a.reps):
        net.forward_device(x.data_ptr(), a.n, a.h, a.w, y.data_ptr(), st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    flops = 2 * 162240 * a.n * a.h * a.w
    return {"kernel": "unet_forward", "variant": a.variant, "conv": a.kernel, "fold": a.fold, "n": a.n, "h": a.h,
            "w": a.w, "ms": ms, "tflops": flops / ms / 1e9, "tiles": tiles}


def trace(a):
    from .render import Renderer
    from .scene import engine_scene
    sc = engine_scene(seed=7)
    r = Renderer(0)
    r.set_scene(sc)
    r.set_bvh_width(a.width)
    r.set_render_tree(a.tree)
    r.set_counting(True)
    c = r.render(spp=a.spp, bounces=a.bounces, accum=False, rgb=False)
    r.set_counting(False)
    rays = c["closest_rays"] + c["shadow_rays"]
    out = {"kernel": "trace", "spp": a.spp, "width": a.width, "tree": r.render_tree(), "rays": rays,
           "nodes_per_ray": c["node_fetches"] / rays, "tris_per_ray": c["tri_tests"] / rays}
    if hasattr(r, "stack_bound"):
        out["stack_bound"] = r.stack_bound()
    sweep = {}
    if a.l2win:
        r.set_l2_window(True)
        out["l2_window"] = True
    for top in (int(x) for x in str(a.top).split(",")):
        if hasattr(r, "set_top_records"):
            r.set_top_records(top)
        for qu in (int(x) for x in str(a.quorum).split(",")):
            r.set_leaf_quorum(qu)
            for th in (int(x) for x in str(a.refill).split(",")):
                r.set_refill_threshold(th)
                r.render(spp=a.spp, bounces=a.bounces, accum=False, rgb=False)
                ms = [r.render(spp=a.spp, bounces=a.bounces, accum=False, rgb=False)["kernel_ms"]
                      for _ in range(a.reps)]
                sweep[f"refill={th},quorum={qu},top={top}"] = {"ms": ms, "mrays_per_s": rays / min(ms) / 1e3}
    if len(sweep) == 1:
        (k, v), = sweep.items()
        out.update(schedule=k, **v)
    else:
        out["schedule"] = sweep
    return out


def bvh(a):
    """LBVH build: device-resident (lg_build_bvh_device, CUDA events) and
    host in/out (lg_build_bvh, wall clock incl. the 105 MB upload/download)."""
    import ctypes as C
    import time

    import torch

    from . import _ffi
    from .render import build_bvh
    from .scene import engine_scene
    sc = engine_scene(seed=7)
    n = sc.n_tris
    d_tris = torch.from_numpy(sc.tris.view(np.uint8).copy()).cuda()
    d_out = torch.empty_like(d_tris)
    d_nodes = torch.empty((2 * n - 1) * 40, dtype=torch.uint8, device="cuda")
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    cnt = C.c_int32(0)
    st = torch.cuda.current_stream()
    L = _ffi.lib()

    def dev_build():
        _ffi.check(L.lg_build_bvh_device(C.c_void_p(d_tris.data_ptr()), n, C.c_void_p(d_nodes.data_ptr()),
                                         C.byref(cnt), C.c_void_p(d_perm.data_ptr()), C.c_void_p(d_out.data_ptr()),
                                         C.c_void_p(st.cuda_stream)))

    for _ in range(3):
        dev_build()
    torch.cuda.synchronize()
    dev_ms = []
    for _ in range(a.reps):
        e0, e1 = _events(torch)
        e0.record(st)
        dev_build()
        e1.record(st)
        torch.cuda.synchronize()
        dev_ms.append(e0.elapsed_time(e1))
    build_bvh(sc.tris)
    host_ms = []
    for _ in range(a.reps):
        t0 = time.perf_counter()
        build_bvh(sc.tris)
        host_ms.append((time.perf_counter() - t0) * 1e3)
    return {"kernel": "lbvh", "triangles": n, "nodes": cnt.value, "device_ms": dev_ms, "host_io_ms": host_ms}


def batch(a):
    """Orbit poses of the engine scene: one batched launch (lg_render_batch,
    graph-replayed) against one launch per frame, device time per frame."""
    from .render import Renderer
    from .scene import ENGINE_CENTER, engine_scene, orbit_poses
    sc = engine_scene(seed=7)
    r = Renderer(0)
    r.set_scene(sc)
    cams = [sc.camera.look_at(p, t) for p, t in orbit_poses(a.poses, seed=11, center=ENGINE_CENTER)]
    n = len(cams)
    spps, bounces = [a.spp] * n, [a.bounces] * n
    tuned = None
    if a.tune:
        # the persistent launch's occupancy and schedule, tuned on the first pose
        bps, _ = r.autotune(camera=cams[0], spp=a.spp, bounces=a.bounces)
        refill, quorum, _ = r.autotune_schedule(camera=cams[0], spp=a.spp, bounces=a.bounces)
        tuned = {"blocks_per_sm": bps, "refill": refill, "quorum": quorum}
    r.render_batch(cams, spps, bounces)  # capture
    _, ms = r.render_batch(cams, spps, bounces)
    sep = [r.render(camera=c, spp=a.spp, bounces=a.bounces, accum=False, rgb=False)["kernel_ms"] for c in cams]
    out = {"kernel": "trace (batched)", "poses": n, "spp": a.spp, "bounces": a.bounces, "tuned": tuned,
           "batch_ms_per_frame": float(ms.sum()) / n, "separate_ms_per_frame": float(np.sum(sep)) / n}
    out["speedup"] = out["separate_ms_per_frame"] / out["batch_ms_per_frame"]
    r.close()
    return out


def train(a):
    """UNet training steps at n x h x w (random crops stand in: the cost does not depend on the values): the
    synchronous step (lg_unet_train_step) and the queued one (lg_unet_train_step_async), wall time per step."""
    import time

    import torch

    from .unet import UNet
    net = UNet(variant=a.variant)
    net.set_params(np.random.default_rng(5).normal(0, 0.02, net.n_params).astype(np.float32))
    x = torch.rand((a.n, 3, a.h, a.w), device="cuda")
    t = torch.rand((a.n, 3, a.h, a.w), device="cuda")
    out = {"kernel": "unet_train_step", "variant": a.variant, "n": a.n, "h": a.h, "w": a.w}
    for _ in range(3):
        net.train_step(x.data_ptr(), t.data_ptr(), a.n, a.h, a.w, 1e-4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.reps):
        net.train_step(x.data_ptr(), t.data_ptr(), a.n, a.h, a.w, 1e-4)
    torch.cuda.synchronize()
    out["sync_ms"] = (time.perf_counter() - t0) / a.reps * 1e3
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        t0 = time.perf_counter()
        for _ in range(a.reps):
            net.train_step_async(x.data_ptr(), t.data_ptr(), a.n, a.h, a.w, 1e-4, 0, s.cuda_stream)
        s.synchronize()
        out["async_ms"] = (time.perf_counter() - t0) / a.reps * 1e3
    net.sync()
    net.close()
    return out


def setup(a):
    """lg_renderer_set_scene on the engine scene from pinned host memory (upload, device LBVH, render tree,
    records), wall time per call."""
    import time

    import torch

    from . import _ffi
    from .render import Renderer
    from .scene import Scene, engine_scene
    sc = engine_scene(seed=7)
    pinned = torch.empty(sc.tris.nbytes, dtype=torch.uint8, pin_memory=True).numpy()
    pinned[:] = sc.tris.view(np.uint8).ravel()
    scp = Scene(sc.camera, sc.sun, pinned.view(_ffi.TRI_DTYPE), sc.mat_albedo, sc.mat_emissive, sc.points)
    r = Renderer(0)
    r.set_scene(scp)
    ms = []
    for _ in range(a.reps):
        t0 = time.perf_counter()
        r.set_scene(scp)
        torch.cuda.synchronize()
        ms.append((time.perf_counter() - t0) * 1e3)
    r.close()
    return {"kernel": "set_scene", "triangles": sc.n_tris, "ms": ms}


def membench(a):
    """Read bandwidth of the L2 (buffers of 8-96 MB, L2-only loads) and of L1
    (every block re-reading a 16 KB region), lg_measure_read_bandwidth."""
    import ctypes as C

    from . import _ffi
    out = {"kernel": "membench", "l2_gbs": {}, "l1_gbs": {}}
    g = C.c_double(0)
    for mb in (8, 16, 32, 48, 64, 96):
        _ffi.check(_ffi.lib().lg_measure_read_bandwidth(0, 2, mb << 20, 40, C.byref(g)))
        out["l2_gbs"][f"{mb}MB"] = g.value
    for kb in (4, 16, 32):
        _ffi.check(_ffi.lib().lg_measure_read_bandwidth(0, 1, kb << 10, 400, C.byref(g)))
        out["l1_gbs"][f"{kb}KB"] = g.value
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["unet", "trace", "bvh", "batch", "membench", "train", "setup"])
    ap.add_argument("--poses", type=int, default=50)
    ap.add_argument("--kernel", default="default", choices=["default", "single", "resident", "rows4", "dyp4", "dyp8", "autotune"],
                    help="unet: default tiles, the one-tile-per-CTA conv kernel, resident weights for the "
                         "single-block layers, or autotuned tiles")
    ap.add_argument("--n", type=int, default=1)
    ap.add_argument("--fold", type=int, default=1, help="unet: folded upsampling in u3a/u2a/u1a (1/0)")
    ap.add_argument("--variant", default="ref", choices=["ref", "hdr"],
                    help="unet: reference network, or the HDR one (ReLU, bilinear upsampling, log1p in / expm1 out)")
    ap.add_argument("--h", type=int, default=864)
    ap.add_argument("--w", type=int, default=1728)
    ap.add_argument("--spp", type=int, default=8)
    ap.add_argument("--bounces", type=int, default=2)
    ap.add_argument("--width", type=int, default=4)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--refill", default="12", help="trace: refill threshold(s), comma-separated")
    ap.add_argument("--quorum", default="12", help="trace: leaf quorum(s), comma-separated")
    ap.add_argument("--top", default="0", help="trace: top records kept in shared memory, comma-separated")
    ap.add_argument("--l2win", type=int, default=0, help="trace: persisting-L2 window over the BVH records (1/0)")
    ap.add_argument("--tune", type=int, default=1, help="batch: autotune the launch and schedule first (1/0)")
    ap.add_argument("--tree", default="ploc_tris", choices=["ploc", "buildbvh", "ploc_tris"], help="trace: render tree")
    a = ap.parse_args(argv)
    print(json.dumps({"unet": unet, "trace": trace, "bvh": bvh, "batch": batch, "membench": membench, "train": train,
                      "setup": setup}[a.what](a)))


if __name__ == "__main__":
    main()
