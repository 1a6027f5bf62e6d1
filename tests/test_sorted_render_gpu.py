"""The ray-sorted render (lg_render_sorted; the reference's RenderSceneCUDASorted,
src/pathtracer.cu:431-547, 759-909, behind `cuda_ref --sort`).

Parity: against the reference's own sorted kernels compiled for sm_100a
(oracle/_ref: gen_primary_kernel, thrust::sort_by_key, trace_and_bounce_kernel,
launched as RenderSceneCUDASorted launches them) on the same BVH and
triangles, with the render bar of the project: >= 99.9% of pixels with every
channel within 1e-3 relative (+1e-6 absolute).  The reference draws every
bounce direction from the RNG state of the ray's sorted slot, so its image
depends on the exact sort order; a ray whose direction key differed in one
bit would move other rays' slots.  Equal keys need the same directions, which
the shared FP32 expressions give.

Also: the drop-in CLI path -- the reference's unchanged src/main.cpp linked
against liblumina.so (built by oracle/Makefile into oracle/_ref/) -- renders
the same PNG as this repository's cuda_ref, plain and with --sort."""
import pathlib
import subprocess

import numpy as np
import pytest

import lumina
import oracle as O

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parent.parent
REF_MAIN = ROOT / "oracle" / "_ref" / "cuda_ref_main"
OUR_CLI = ROOT / "luminagi-cudaref_b200" / "bin" / "cuda_ref"


def match_fraction(a, b, rel=1e-3, abs_=1e-6):
    close = np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + abs_
    return float(close.all(axis=2).mean())


def ours_sorted(scene, nodes, tris, spp, bounces, width=4, sort=True, camera=None):
    sc = lumina.Scene(scene.camera, scene.sun, tris, scene.mat_albedo, scene.mat_emissive, scene.points)
    with lumina.Renderer(0) as r:
        r.set_scene_bvh(sc, nodes)
        r.set_bvh_width(width)
        return r.render_sorted(camera=camera, spp=spp, bounces=bounces, sort=sort)


@pytest.mark.parametrize("width", [4, 2])
@pytest.mark.parametrize("spp,bounces", [(1, 0), (4, 1), (4, 2)])
def test_sorted_vs_reference_sorted_gpu(box_scene, spp, bounces, width):
    if not O.ref_available():
        pytest.skip("reference oracle not built")
    nodes, tris, _, _ = O.oracle_build_bvh(box_scene.tris)
    ours = ours_sorted(box_scene, nodes, tris, spp, bounces, width=width)
    ref_acc, ref_rgb, _ = O.ref_render_gpu(box_scene, nodes, tris, spp, bounces, sorted_path=True)
    f = match_fraction(ours["accum"], ref_acc)
    assert f >= 0.999, f
    assert float((ours["rgb"] == ref_rgb).all(axis=2).mean()) >= 0.999


def test_sorted_engine_small_vs_reference_sorted_gpu(small_engine_scene):
    if not O.ref_available():
        pytest.skip("reference oracle not built")
    sc = small_engine_scene
    nodes, tris, _, _ = O.oracle_build_bvh(sc.tris)
    ours = ours_sorted(sc, nodes, tris, 8, 2)
    ref_acc, _, _ = O.ref_render_gpu(sc, nodes, tris, 8, 2, sorted_path=True)
    f = match_fraction(ours["accum"], ref_acc)
    print(f"sorted path, small engine scene 8 spp 2 bounces: {f:.6%} of pixels within 1e-3")
    assert f >= 0.999, f


def test_sort_only_reorders_work_without_bounces(box_scene):
    """With no bounce, no draw follows the camera jitter, so the sort cannot
    change the image: sorted and unsorted give the same accumulator bits, and
    the persistent trace kernel (one sample: its chunk seed is the sample
    seed) the same image within the render bar (the two kernels may contract
    the same FP32 expressions into FMAs differently)."""
    with lumina.Renderer(0) as r:
        r.set_scene(box_scene)
        a = r.render_sorted(spp=1, bounces=0)["accum"]
        b = r.render_sorted(spp=1, bounces=0, sort=False)["accum"]
        c = r.render(spp=1, bounces=0)["accum"]
    assert np.array_equal(a, b)
    assert match_fraction(a, c) >= 0.9999


def test_sorted_counts_and_estimator(box_scene):
    """Sorted and unsorted wavefronts trace different rays (the slot RNG) but
    the same estimator: their mean radiance agrees within a few percent, and
    counting reports every camera ray of every sample."""
    with lumina.Renderer(0) as r:
        r.set_scene(box_scene)
        r.set_counting(True)
        a = r.render_sorted(spp=8, bounces=2)
        b = r.render_sorted(spp=8, bounces=2, sort=False)
    W, H = int(box_scene.camera.width), int(box_scene.camera.height)
    assert a["closest_rays"] >= 8 * W * H and a["shadow_rays"] > 0
    ma, mb = float(a["accum"].mean()), float(b["accum"].mean())
    assert abs(ma - mb) <= 0.03 * max(ma, mb), (ma, mb)


@pytest.mark.parametrize("wt", [False, True])
def test_staged_bounces_match_one_thread_per_ray(small_engine_scene, wt):
    """A bounce runs as four launches (closest hits on persistent warps,
    shading and shadow rays, occlusion on persistent warps, pixel update and
    next rays) unless counting is on, when the one-thread-per-ray launch runs
    and counts.  Both compute the same expressions in the same order: the
    images agree under the render bar (closest hits differ only on exact ties),
    sorted and unsorted, with either intersection test."""
    with lumina.Renderer(0) as r:
        r.set_scene(small_engine_scene)
        r.set_intersection("watertight" if wt else "mt")
        for sort in (True, False):
            r.set_counting(True)
            a = r.render_sorted(spp=4, bounces=2, sort=sort)["accum"]
            r.set_counting(False)
            b = r.render_sorted(spp=4, bounces=2, sort=sort)["accum"]
            assert a.any()
            assert match_fraction(a, b) >= 0.999


def test_many_lights_trace_one_ray_per_thread(box_scene):
    """Scenes with more than 8 lights (the sun and the point lights) keep the
    one-thread-per-ray bounce, which needs no per-light buffers: the frame
    renders and matches the counting launch bit for bit (same kernel)."""
    pts = np.concatenate([box_scene.points] * 9)
    sc = lumina.Scene(box_scene.camera, box_scene.sun, box_scene.tris, box_scene.mat_albedo, box_scene.mat_emissive,
                      pts)
    with lumina.Renderer(0) as r:
        r.set_scene(sc)
        b = r.render_sorted(spp=2, bounces=1)["accum"]
        r.set_counting(True)
        a = r.render_sorted(spp=2, bounces=1)
    assert a["shadow_rays"] > 0 and b.any()
    assert np.array_equal(a["accum"], b)


def _png(path):
    from PIL import Image
    return np.asarray(Image.open(path).convert("RGB"))


@pytest.mark.parametrize("sort", [False, True])
def test_reference_main_linked_renders_like_cuda_ref(tmp_path, sort):
    """The reference's src/main.cpp, linked against liblumina.so, and this
    repository's cuda_ref give the same image of the same scene file."""
    if not REF_MAIN.exists():
        pytest.skip("reference CLI not built against the library (oracle/Makefile)")
    sc = lumina.box_scene(1, width=160, height=80)
    scene_dir = tmp_path / "scenes"
    scene_dir.mkdir()
    sc.save_json(str(scene_dir / "box.json"))
    extra = ["--sort"] if sort else []
    outs = []
    for exe, name in ((REF_MAIN, "ref.png"), (OUR_CLI, "ours.png")):
        png = tmp_path / name
        p = subprocess.run([str(exe), str(scene_dir / "box.json"), str(png), "--spp", "4", "--bounces", "1"] + extra,
                           capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, (exe, p.stdout[-2000:], p.stderr[-2000:])
        assert ("kernel (sorted):" in p.stdout) == sort, p.stdout
        outs.append(_png(png))
    assert outs[0].shape == (80, 160, 3)
    assert np.array_equal(outs[0], outs[1])
