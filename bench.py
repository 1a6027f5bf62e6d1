"""Benchmark: the plain path-traced frame of the engine-scale scene on B200.

Workload (one "step"): one 1728x864 frame of the 1,050,972-triangle seeded
engine-scale scene at 64 spp and 2 bounces (the reference's headline render
configuration), traced by liblumina's kernels.  Reported as Mrays/s (closest-
hit + shadow rays actually traced, counted exactly by the kernel in a separate
counting pass) with ms/frame alongside.

  value     device-resident: scene and BVH already in HBM, K frames timed with
            CUDA events on the launching stream.
  e2e       through the C ABI from host buffers: triangle upload from pinned
            memory, device LBVH build, render, tonemap and the 8-bit image read
            back, every step.
  roofline  algorithmic bytes of the trace kernel (64 B per 4-wide BVH
            record, both 32-byte halves as loaded; 48 B per triangle test;
            8 B per leaf-table entry; as counted) over its event-timed
            duration, against the L2 read bandwidth measured in this run
            (lg_measure_read_bandwidth: a 64 MB buffer, L2-only loads).  The
            hot arrays (records ~22 MB, triangle records ~67 MB) stay
            L2-resident across frames: DRAM moves ~8 B per ray.  L1 and HBM
            fractions ride along.
  ref_gpu   the reference's accumulate_kernel compiled for sm_100a
            (oracle/_ref) on the same frame and BVH, timed with CUDA events
            as RenderSceneCUDA times it: the reference design on this GPU.
  sorted    the ray-sorted render (RenderSceneCUDASorted semantics) of the
            same frame: this library with and without its ray sort, and the
            reference's sorted kernels on this GPU.
  cpu_baseline  the reference's own trace code (oracle/_ref, compiled from its
            sources for the host) with OpenMP on all host cores, on a fixed
            sample of rows (every CPU_ROW_STEP-th row; the reference arm uses
            the same rows); rays counted by the oracle on the same rows.
  denoise   8 spp + UNet against plain 256 spp on the same frame (device
            time), with the trained weights in lumina/data: PSNR/SSIM of both
            and of the 8-spp input against a 1024-spp FP64 judge on an orbit
            pose held out of training; and the denoiser alone (reference and
            HDR networks, batch 1 and 8) in TFLOP/s against the dense BF16
            peak.
  ingest    scene-file load times: this library on scene.json and on the
            binary scene file, and the reference's LoadSceneJSON on the same
            JSON (host only).
  batched   the 50 orbit poses of the engine scene in one graph-replayed
            persistent launch (lg_render_batch) against one launch per pose,
            device ms per frame, at 8 spp (all 50) and 256 spp (the first 4).

--impl reference times only that CPU path (the reference renderer has no
other CPU path) on the same rows, over the reference's own BuildBVH, and
prints its line.  Multi-GPU: replicas (each rank renders
its own frame; no collective), value summed over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "luminagi-cudaref_b200"))

import numpy as np  # noqa: E402

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# DRAM bytes (read + write) per traced ray of trace_kernel, from one ncu capture
# of an 8-spp engine frame: 427.7 MB + 37.8 MB / 65,366,791 rays; traffic
# scales with rays.
TRACE_DRAM_BYTES_PER_RAY = (427703296 + 37808384) / 65366791
# Bytes one traversal step loads from a BVH record: both 32-byte halves of a
# 4-wide record (grid origin, steps, 24 one-byte planes, four links), or the
# whole 64-byte 2-wide record.
RECORD_BYTES = {4: 64, 2: 64}
# Rows of the CPU sample: every CPU_ROW_STEP-th row of the frame, the same in
# the cpu_baseline leg and the reference arm.
CPU_ROW_STEP = 16
# Multiply-adds per output pixel of the denoiser (14 3x3 convolutions and the 1x1 tail; ml/train.py's UNet).
UNET_MAC_PER_PIXEL = 162240
# Local-memory (stack and spill) bytes per traced ray of trace_kernel, from the
# same capture: (806.4 M load + 911.3 M store sectors) x 32 B / rays.
TRACE_LOCAL_BYTES_PER_RAY = (806358764 + 911343284) * 32 / 65366791
# Denoiser weights trained by this library on the engine scene (lumina.surrogate, the
# 120-epoch recipe with 24 crops per image per epoch; FP16 copy of the best-validation
# parameters, with the indices of the poses held out of training).
PRETRAINED = ROOT / "luminagi-cudaref_b200" / "lumina" / "data" / "unet_engine_long.npz"
# L2 probe: buffer size and passes; 64 MB gave the highest read bandwidth of the
# sizes tried (8-96 MB), the conservative denominator.
L2_PROBE_BYTES = 64 << 20
L1_PROBE_BYTES = 16 << 10


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--bounces", type=int, default=2)
    ap.add_argument("--scene", default="engine", choices=["engine", "box"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-denoise", action="store_true", help="skip the 8spp+UNet vs 256spp timing")
    ap.add_argument("--cpu-row-step", type=int, default=CPU_ROW_STEP,
                    help="CPU sample: every N-th row of the frame (cpu_baseline and the reference arm)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference kernels on this GPU (ref_gpu, sorted)")
    ap.add_argument("--no-ingest", action="store_true", help="skip the scene-file load timing")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched orbit-pose frames (one graph-replayed launch against one launch per pose)")
    return ap.parse_args()


def make_scene(kind):
    import lumina
    if kind == "box":
        return lumina.box_scene(1), "box_20k_512x256"
    return lumina.engine_scene(seed=7), "engine_1.05M_1728x864"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        fd, name = tempfile.mkstemp(prefix="lumina_clocks_", suffix=".csv")
        os.close(fd)
        self.path = pathlib.Path(name)

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        text = self.path.read_text()
        try:
            self.path.unlink()
        except OSError:
            pass
        for line in text.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def sample_rays(scene, nodes, tris, spp, bounces, step):
    """Rays (closest + shadow) the frame's sampled rows trace, counted by the
    oracle on the same paths (the counts are deterministic)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    _, cnt = O.oracle_render(scene, nodes, tris, spp, bounces, row_start=0, row_step=step,
                             threads=os.cpu_count() or 1)
    return cnt["closest_rays"] + cnt["shadow_rays"]


def cpu_baseline(scene, nodes, tris, spp, bounces, step=CPU_ROW_STEP, rays=None):
    """The reference's trace code on all host cores over every step-th row,
    as Mrays/s and scaled to a full frame."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    H = int(scene.camera.height)
    use_ref = O.ref_available()
    threads = os.cpu_count() or 1
    run = O.ref_trace_cpu if use_ref else (lambda *a, **k: O.oracle_render(*a, **k)[0])
    if rays is None:
        rays = sample_rays(scene, nodes, tris, spp, bounces, step)
    t = time.perf_counter()
    run(scene, nodes, tris, spp, bounces, row_start=0, row_step=step, threads=threads)
    dt = time.perf_counter() - t
    n_rows = len(range(0, H, step))
    return {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": threads,
            "kind": "reference" if use_ref else "port",
            "sample": f"every {step}th row ({n_rows} of {H} rows) of the same frame, {spp} spp, {bounces} bounces; "
                      f"{rays} rays in {dt:.2f} s",
            "ms_per_frame_scaled": dt * 1e3 * H / n_rows}


def ingest_timing(scene, with_reference: bool):
    """Scene-file load times (host): this library's loader on the scene written
    as scene.json and as the binary scene file, best of 3 each, and the
    reference's LoadSceneJSON (oracle/_ref) on the same JSON once.  Files go to
    a temporary directory and are removed afterwards."""
    import ctypes as C
    import tempfile
    from lumina import _ffi
    out = {"triangles": scene.n_tris, "threads": os.cpu_count()}
    with tempfile.TemporaryDirectory() as d:
        pj, pb = os.path.join(d, "scene.json"), os.path.join(d, "scene.lgscene")
        scene.save_json(pj)
        scene.save_bin(pb)
        out["json_bytes"], out["bin_bytes"] = os.path.getsize(pj), os.path.getsize(pb)
        L = _ffi.lib()
        for key, path in (("json_s", pj), ("bin_s", pb)):
            best = float("inf")
            for _ in range(3):
                h = C.c_void_p()
                t0 = time.perf_counter()
                _ffi.check(L.lg_scene_load_json(path.encode(), 0, 0, C.byref(h)))
                best = min(best, time.perf_counter() - t0)
                L.lg_scene_destroy(h)
            out[key] = best
        if with_reference:
            try:
                sys.path.insert(0, str(ROOT / "oracle"))
                import oracle as O
                # the reference loader prints its summary with printf: keep fd 1 clean
                sys.stdout.flush()
                saved = os.dup(1)
                devnull = os.open(os.devnull, os.O_WRONLY)
                os.dup2(devnull, 1)
                try:
                    t0 = time.perf_counter()
                    ok = O.ref_load_scene(pj) is not None
                    dt = time.perf_counter() - t0
                finally:
                    os.dup2(saved, 1)
                    os.close(saved)
                    os.close(devnull)
                out["reference_json_s"] = dt if ok else None
                out["speedup_json"] = out["reference_json_s"] / out["json_s"] if ok else None
            except Exception as e:  # the reference build is test infrastructure; report, don't fail
                out["reference_json_s"] = None
                out["reference_error"] = str(e)
    return out


def max_over_ranks(v: float, dist, device="cpu") -> float:
    """The slowest rank's time (every rank takes the same collective steps)."""
    if not dist:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(rays_per_frame: int, steps: int, world: int, ms_total_max: float) -> float:
    """Whole-job Mrays/s of `world` replicas each rendering `steps` frames, timed by the slowest rank."""
    return rays_per_frame * steps * world / (ms_total_max / 1e3) / 1e6


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def reference_designs_on_gpu(scene, spp, bounces, ours_kernel_ms, r):
    """The reference's kernels compiled for sm_100a (oracle/_ref) on the same
    frame, over the reference's own BuildBVH: accumulate_kernel (the plain
    render) and the ray-sorted path, each timed with CUDA events around its
    launches as the reference times them; plus this library's sorted render
    with and without its ray sort.  Second of two runs each."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    if not O.ref_available():
        return None, None
    nodes, tris = O.ref_build_bvh(scene.tris)
    plain = [O.ref_render_gpu(scene, nodes, tris, spp, bounces)[2] for _ in range(2)][-1]
    ref_gpu = {"ms_per_frame": plain, "ours_kernel_ms": ours_kernel_ms, "speedup": plain / ours_kernel_ms,
               "what": "reference accumulate_kernel + tonemap_kernel, sm_100a build, same frame and BVH"}
    srt = [O.ref_render_gpu(scene, nodes, tris, spp, bounces, sorted_path=True)[2] for _ in range(2)][-1]
    ours = [r.render_sorted(spp=spp, bounces=bounces)["kernel_ms"] for _ in range(2)][-1]
    ours_nosort = [r.render_sorted(spp=spp, bounces=bounces, sort=False)["kernel_ms"] for _ in range(2)][-1]
    sorted_cmp = {"ref_ms_per_frame": srt, "ours_ms_per_frame": ours, "ours_ms_without_ray_sort": ours_nosort,
                  "speedup_vs_ref": srt / ours,
                  "what": "RenderSceneCUDASorted semantics (per-sample seeding, rays sorted by direction "
                          "between bounces, no Russian roulette); the reference's sorted kernels vs lg_render_sorted"}
    return ref_gpu, sorted_cmp


def batched_poses(r, scene, bounces, poses_8=50, poses_256=4):
    """Orbit poses of the engine scene (radius 15-25 m, height 2-8 m, looking at
    the scene centre; the 50 poses the denoiser's data come from) rendered in one
    persistent trace launch replayed from a CUDA graph (lg_render_batch) against
    one launch per pose (lg_render), device time per frame.  8 spp over all 50
    poses; 256 spp over the first `poses_256` of them (the per-frame cost does
    not depend on how many poses share the launch, and 50 such frames would take
    almost a minute).  The batched time includes the graph's accumulator clears
    and per-frame tonemaps; the separate one is the trace kernel alone."""
    from lumina.scene import ENGINE_CENTER, orbit_poses
    poses = orbit_poses(50, seed=11, center=ENGINE_CENTER)
    out = {"what": "orbit poses in one graph-replayed persistent launch vs one launch per pose, device ms per frame"}
    for spp, n in ((8, poses_8), (256, poses_256)):
        cams = [scene.camera.look_at(p, t) for p, t in poses[:n]]
        r.render_batch(cams, [spp] * n, [bounces] * n)  # the first call captures the graph
        _, ms = r.render_batch(cams, [spp] * n, [bounces] * n)
        sep = [r.render(camera=c, spp=spp, bounces=bounces, accum=False, rgb=False)["kernel_ms"] for c in cams]
        b, s = float(ms.sum()) / n, float(np.sum(sep)) / n
        out[f"spp{spp}"] = {"poses": n, "bounces": bounces, "batch_ms_per_frame": b, "separate_ms_per_frame": s,
                            "speedup": s / b}
    return out


def main():
    args = parse_args()
    world, rank, local, dist = dist_setup(args)
    peaks, peak_kind = load_peaks()
    scene, workload = make_scene(args.scene)
    cfg = {"workload": workload, "triangles": scene.n_tris, "width": int(scene.camera.width),
           "height": int(scene.camera.height), "spp": args.spp, "bounces": args.bounces,
           "rng": "xorshift32 per (pixel, chunk of 8 samples), reference seeding",
           "l2": "no flush: the BVH records (~22 MB) and triangle records (~67 MB) stay L2-resident across "
                 "frames, as they would across a renderer's frames; DRAM moves ~8 B per ray",
           "parallelism": f"replicas x{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        nodes, tris = O.ref_build_bvh(scene.tris)  # the reference's own BuildBVH
        rays = sample_rays(scene, nodes, tris, args.spp, args.bounces, args.cpu_row_step)
        vals = []
        for i in range(args.warmup + args.steps):
            b = cpu_baseline(scene, nodes, tris, args.spp, args.bounces, args.cpu_row_step, rays)
            if i >= args.warmup:
                vals.append(b)
        v = statistics.median([b["value"] for b in vals])
        ms = statistics.median([b["ms_per_frame_scaled"] for b in vals])
        b = vals[-1]
        line = {"impl": "reference", "metric": "Mrays/s (plain render; ms/frame alongside)", "value": v,
                "unit": "Mrays/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded procedural scene)", "config": cfg,
                "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": b["cores"], "kind": b["kind"],
                                 "sample": b["sample"]},
                "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "ms_per_step_note": "each step traces the sampled rows; ms_per_step is that time scaled to the "
                                    "full frame"}
        print(json.dumps(line))
        return

    import ctypes as C

    import torch
    import lumina
    from lumina import _ffi

    torch.cuda.set_device(local)
    dev = local
    # Cache read bandwidths of this GPU (the trace kernel's roofline denominators).
    l2_gbs, l1_gbs = C.c_double(0), C.c_double(0)
    _ffi.check(_ffi.lib().lg_measure_read_bandwidth(dev, 2, L2_PROBE_BYTES, 40, C.byref(l2_gbs)))
    _ffi.check(_ffi.lib().lg_measure_read_bandwidth(dev, 1, L1_PROBE_BYTES, 400, C.byref(l1_gbs)))
    r = lumina.Renderer(dev)
    r.set_scene(scene)
    nodes_dev, tris_dev = r.get_bvh()
    cfg["trace"] = {"records": "4-wide, 8-bit quantized planes, 64 B", "render_tree": r.render_tree(),
                    "refill_threshold": r.refill_threshold(), "leaf_quorum": r.leaf_quorum()}

    # counting pass (not timed)
    r.set_counting(True)
    c = r.render(spp=args.spp, bounces=args.bounces, accum=False, rgb=False)
    r.set_counting(False)
    rays = c["closest_rays"] + c["shadow_rays"]
    algo_bytes = RECORD_BYTES[4] * c["node_fetches"] + 48 * c["tri_tests"] + 8 * c["leaf_fetches"]

    cam = scene.camera.to_c()
    opts = _ffi.LgRenderOpts(args.spp, args.bounces, 0, 0)
    stream = torch.cuda.current_stream(dev)

    def step_device():
        _ffi.check(_ffi.lib().lg_render_device(r._h, C.byref(cam), C.byref(opts), C.c_void_p(stream.cuda_stream),
                                               None, None, None))

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step_device()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    ms_total = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{dev}")
    ms_step = ms_total / args.steps
    value = replica_throughput(rays, args.steps, world, ms_total)

    # kernel-only duration (events around trace + tonemap on the renderer's stream)
    kms = []
    for _ in range(2):
        kms.append(r.render(spp=args.spp, bounces=args.bounces, accum=False, rgb=False)["kernel_ms"])
    kernel_ms = statistics.median(kms)
    achieved = algo_bytes / (kernel_ms / 1e3) / 1e9

    # e2e through the C ABI from pinned host buffers
    pinned = torch.empty(scene.tris.nbytes, dtype=torch.uint8, pin_memory=True).numpy()
    pinned[:] = scene.tris.view(np.uint8).ravel()
    tris_pinned = pinned.view(_ffi.TRI_DTYPE)
    e2e_scene = lumina.Scene(scene.camera, scene.sun, tris_pinned, scene.mat_albedo, scene.mat_emissive,
                             scene.points)
    W, H = int(scene.camera.width), int(scene.camera.height)
    rgb = torch.empty(W * H * 3, dtype=torch.uint8, pin_memory=True).numpy()
    st = _ffi.LgRenderStats()

    def step_e2e():
        d = e2e_scene.desc()
        _ffi.check(_ffi.lib().lg_renderer_set_scene(r._h, C.byref(d)))
        _ffi.check(_ffi.lib().lg_render(r._h, C.byref(cam), C.byref(opts), _ffi.ptr(rgb), None, None, C.byref(st)))

    step_e2e()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    torch.cuda.synchronize(dev)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps, dist, f"cuda:{dev}")
    h2d = scene.tris.nbytes + scene.mat_albedo.nbytes + scene.points.nbytes
    d2h = W * H * 3

    # Headline comparison: 8 spp + UNet denoise vs the plain 256-spp render (device time), and their quality
    # against a 1024-spp FP64 judge on a pose the denoiser was not trained on.
    denoise = None
    if not args.no_denoise and args.scene == "engine":
        net = lumina.UNet()
        trained = PRETRAINED.exists()
        if trained:
            z = np.load(PRETRAINED)
            net.set_params(z["params"].astype(np.float32))
        else:  # the cost of a forward pass does not depend on the values
            net.set_params(np.random.default_rng(0).normal(0, 0.02, net.n_params).astype(np.float32))
        x = torch.empty((1, 3, H, W), device=f"cuda:{dev}")
        y = torch.empty_like(x)
        o8 = _ffi.LgRenderOpts(8, args.bounces, 0, 0)
        o256 = _ffi.LgRenderOpts(256, args.bounces, 0, 0)
        rgbp = C.c_void_p()

        def step_denoised():
            _ffi.check(_ffi.lib().lg_render_device(r._h, C.byref(cam), C.byref(o8), C.c_void_p(stream.cuda_stream),
                                                   C.byref(rgbp), None, None))
            _ffi.check(_ffi.lib().lg_rgb8_to_f32(rgbp, 1, H, W, C.c_void_p(x.data_ptr()),
                                                C.c_void_p(stream.cuda_stream)))
            net.forward_device(x.data_ptr(), 1, H, W, y.data_ptr(), stream.cuda_stream)

        def timed(fn, reps):
            fn()
            torch.cuda.synchronize(dev)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(reps):
                fn()
            a1.record(stream)
            torch.cuda.synchronize(dev)
            return a0.elapsed_time(a1) / reps

        ms_d = timed(step_denoised, 5)
        ms_p = timed(lambda: _ffi.check(_ffi.lib().lg_render_device(
            r._h, C.byref(cam), C.byref(o256), C.c_void_p(stream.cuda_stream), None, None, None)), 1)
        denoise = {"ms_8spp_plus_unet": ms_d, "ms_256spp": ms_p, "speedup": ms_p / ms_d,
                   "weights": "trained (lumina/data/unet_engine_long.npz)" if trained else
                              "random (the cost of a forward pass does not depend on their values)"}
        if trained:
            from lumina import surrogate as S
            from lumina.scene import ENGINE_CENTER, orbit_poses
            pose = int(z["val_idx"][0])
            p_t = orbit_poses(int(z["poses"]), seed=11, center=ENGINE_CENTER)[pose]
            vcam = scene.camera.look_at(*p_t)
            frames = S.eval_frames(r, [vcam], 8, 256, 1024, args.bounces)
            agg, _ = S.evaluate(net, frames)
            denoise["quality"] = {
                "pose": f"orbit pose {pose} of {int(z['poses'])} (held out of training)",
                "judge": "1024 spp, FP64 accumulators", "metric": "PSNR/SSIM of the 8-bit tonemapped images",
                "psnr_8spp": agg["noisy_psnr"], "psnr_8spp_unet": agg["denoised_psnr"],
                "psnr_256spp": agg["clean_psnr"], "ssim_8spp": agg["noisy_ssim"],
                "ssim_8spp_unet": agg["denoised_ssim"], "ssim_256spp": agg["clean_ssim"],
                "gain_db_over_8spp": agg["denoised_psnr"] - agg["noisy_psnr"],
                "db_vs_256spp": agg["denoised_psnr"] - agg["clean_psnr"]}
        net.close()

        # The denoiser alone against the dense BF16 peak (configuration 4): the reference network and the HDR one
        # (ReLU, bilinear upsampling, log1p in / expm1 out) at batch 1 and 8, 1728x864, inputs already on the device.
        def unet_rate(variant, n):
            m = lumina.UNet(variant=variant)
            m.set_params(np.random.default_rng(1).normal(0, 0.02, m.n_params).astype(np.float32))
            xb = torch.rand((n, 3, H, W), device=f"cuda:{dev}")
            yb = torch.empty_like(xb)
            ms = timed(lambda: m.forward_device(xb.data_ptr(), n, H, W, yb.data_ptr(), stream.cuda_stream), 10)
            m.close()
            tf = 2 * UNET_MAC_PER_PIXEL * n * H * W / ms / 1e9
            return {"ms": ms, "tflops": tf, "frac": tf / peaks["bf16_tflops"]}

        denoise["unet"] = {"flop_per_pixel": 2 * UNET_MAC_PER_PIXEL, "peak_tflops": peaks["bf16_tflops"],
                           "peak_source": f"{peak_kind} dense BF16 GEMM, burst",
                           "ref": {"batch1": unet_rate("ref", 1), "batch8": unet_rate("ref", 8)},
                           "hdr": {"batch1": unet_rate("hdr", 1), "batch8": unet_rate("hdr", 8)}}

    traffic = TRACE_DRAM_BYTES_PER_RAY * rays
    roof = {"bound": "l2", "achieved": achieved, "peak": l2_gbs.value, "unit": "GB/s",
            "frac": achieved / l2_gbs.value, "traffic": traffic,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of an 8-spp launch, scaled by rays",
            "peak_source": f"measured in this run: L2 read bandwidth, {L2_PROBE_BYTES >> 20} MB buffer, "
                           "ld.global.cg (lg_measure_read_bandwidth)",
            "l1_peak": l1_gbs.value, "l1_frac": achieved / l1_gbs.value,
            "hbm_peak": peaks["hbm_gbs"], "hbm_frac": achieved / peaks["hbm_gbs"], "hbm_peak_source": peak_kind,
            "dram_bytes_per_ray": TRACE_DRAM_BYTES_PER_RAY, "kernel": "trace_kernel",
            "algorithmic_bytes_per_launch": algo_bytes, "algorithmic_bytes_per_ray": algo_bytes / rays,
            "kernel_ms": kernel_ms,
            "limiter": "instruction issue, not memory (ncu: issue slots 71% busy at 16 of 32 lanes active, "
                       "L1 data pipe 53%; 455 warp instructions per ray)"}
    if TRACE_LOCAL_BYTES_PER_RAY is not None:
        roof["local_bytes_per_ray"] = TRACE_LOCAL_BYTES_PER_RAY
    line = {"metric": "Mrays/s (plain render; ms/frame alongside)", "value": value, "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene)", "config": cfg,
            "rays_per_frame": rays, "ms_per_frame": ms_step,
            "e2e": {"value": rays * world / e2e_s / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_frame": e2e_s * 1e3},
            "roofline": roof,
            "gpu_launches": args.steps * 2,
            "clocks": clk.summary()}
    if denoise:
        line["denoise"] = denoise
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        try:
            ref_gpu, sorted_cmp = reference_designs_on_gpu(scene, args.spp, args.bounces, kernel_ms, r)
            if ref_gpu:
                line["ref_gpu"] = ref_gpu
                line["sorted"] = sorted_cmp
        except Exception as e:  # the oracle libraries are test infrastructure; report, don't fail
            line["ref_gpu"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_batched and args.scene == "engine":
        line["batched"] = batched_poses(r, scene, args.bounces)
    if rank == 0 and world == 1 and not args.no_ingest:
        line["ingest"] = ingest_timing(scene, with_reference=not args.no_cpu_baseline)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(scene, nodes_dev, tris_dev, args.spp, args.bounces, args.cpu_row_step)
        except Exception as e:  # the oracle libraries are test infrastructure; report, don't fail
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    r.close()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
