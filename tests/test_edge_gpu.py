"""Edge cases of the render paths on the device, against the reference's own
kernels compiled for sm_100a (oracle/_ref) where the reference defines the
result:

- image sizes that are not multiples of the 8x4-pixel work tiles, down to one
  pixel, and sample counts that end in a partial chunk of 8 (the reference
  seeds each chunk of 8 samples from its first sample, pathtracer.cu:349, and
  launches the last chunk short, :699-703);
- the ray-sorted render at the same sizes (RenderSceneCUDASorted,
  pathtracer.cu:759-909);
- a scene without triangles: every ray misses, so the accumulators, the image
  and the G-buffer are the miss values.  The reference traverses node 0 of an
  empty array there, so this case has no reference run; the expected values
  are its miss branches (trace_path's `break` on a miss, :305; gbuffer_kernel's
  miss colours, :387-394)."""
import numpy as np
import pytest

import lumina
import oracle as O

pytestmark = pytest.mark.gpu
SIZES = [(1, 1), (13, 7), (37, 29), (300, 9)]


def match_fraction(a, b, rel=1e-3, abs_=1e-6):
    close = np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + abs_
    return float(close.all(axis=2).mean())


def _renderer(scene, nodes, tris):
    sc = lumina.Scene(scene.camera, scene.sun, tris, scene.mat_albedo, scene.mat_emissive, scene.points)
    r = lumina.Renderer(0)
    r.set_scene_bvh(sc, nodes)
    return r


@pytest.mark.parametrize("w,h", SIZES)
def test_ragged_sizes_and_partial_chunks_vs_reference_gpu(box_scene, w, h):
    if not O.ref_available():
        pytest.skip("reference oracle not built")
    nodes, tris, _, _ = O.oracle_build_bvh(box_scene.tris)
    cam = box_scene.camera.copy()
    cam.width, cam.height = w, h
    with _renderer(box_scene, nodes, tris) as r:
        for spp in (3, 13):
            ours = r.render(camera=cam, spp=spp, bounces=2)
            ref_acc, ref_rgb, _ = O.ref_render_gpu(box_scene, nodes, tris, spp, 2, camera=cam)
            assert ours["accum"].shape == (h, w, 3)
            # fewer than 1,000 pixels: the 99.9% bar means every pixel
            assert match_fraction(ours["accum"], ref_acc) >= 0.999
            assert float((ours["rgb"] == ref_rgb).all(axis=2).mean()) >= 0.999


@pytest.mark.parametrize("w,h", SIZES)
def test_ragged_sizes_sorted_vs_reference_sorted_gpu(box_scene, w, h):
    if not O.ref_available():
        pytest.skip("reference oracle not built")
    nodes, tris, _, _ = O.oracle_build_bvh(box_scene.tris)
    cam = box_scene.camera.copy()
    cam.width, cam.height = w, h
    with _renderer(box_scene, nodes, tris) as r:
        ours = r.render_sorted(camera=cam, spp=3, bounces=2)
    ref_acc, ref_rgb, _ = O.ref_render_gpu(box_scene, nodes, tris, 3, 2, camera=cam, sorted_path=True)
    assert match_fraction(ours["accum"], ref_acc) >= 0.999
    assert float((ours["rgb"] == ref_rgb).all(axis=2).mean()) >= 0.999


def test_scene_without_triangles_renders_misses(box_scene):
    empty = box_scene.tris[:0]
    sc = lumina.Scene(box_scene.camera, box_scene.sun, empty, box_scene.mat_albedo, box_scene.mat_emissive,
                      box_scene.points)
    cam = box_scene.camera.copy()
    cam.width, cam.height = 37, 29
    with lumina.Renderer(0) as r:
        r.set_scene(sc)
        assert r.get_bvh()[0].shape[0] == 0
        for width in (4, 2):
            r.set_bvh_width(width)
            o = r.render(camera=cam, spp=13, bounces=2)
            assert not o["accum"].any() and not o["rgb"].any()
            s = r.render_sorted(camera=cam, spp=3, bounces=2)
            assert not s["accum"].any() and not s["rgb"].any()
        alb, nrm, wp = r.gbuffer(camera=cam)
        assert not alb.any() and not wp.any()
        assert (nrm == np.array([128, 128, 255], np.uint8)).all()
