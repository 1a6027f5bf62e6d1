"""Diffuse textures (load_texture_to_device + sample_albedo, reference
pathtracer.cu:553-579, 274-282) against the reference kernels with the
reference's own texture objects, on the same BVH, triangles and PNG files."""
import subprocess

import numpy as np
import pytest

import lumina
import oracle as O
import pngenc
from lumina import _ffi

pytestmark = pytest.mark.gpu
REL, ABS = 1e-3, 1e-6


@pytest.fixture(scope="module")
def textured(tmp_path_factory):
    """Box scene with a checker on the walls and a noise texture on the
    spheres; uvs stretched to [-0.7, 2.3] so wrapping is exercised."""
    root = tmp_path_factory.mktemp("assets")
    (root / "tex").mkdir()
    yy, xx = np.mgrid[0:64, 0:48]
    checker = np.where(((yy // 8) + (xx // 8)) % 2 == 0, 220, 40)
    chk = np.stack([checker, checker // 2 + 60, 255 - checker], -1)
    (root / "tex" / "checker.png").write_bytes(pngenc.encode(chk, 2, 8))
    noise = np.random.default_rng(5).integers(0, 65536, (17, 29, 4))
    (root / "tex" / "noise.png").write_bytes(pngenc.encode(noise, 6, 16, interlace=True))
    sc = lumina.box_scene(3, width=192, height=96, sphere_subdiv=3)
    sc.tris["uv"] = sc.tris["uv"] * np.float32(3.0) - np.float32(0.7)
    n_mats = len(sc.mat_albedo)
    sc.textures = ["tex/checker.png" if m < n_mats - 4 else "tex/noise.png" for m in range(n_mats)]
    sc.textures[1] = "tex/missing.png"
    scenes = root / "scenes"
    scenes.mkdir()
    sc.save_json(scenes / "scene.json")
    return sc, root


def _setup(sc, root, width):
    nodes, tris, _, _ = O.oracle_build_bvh(sc.tris)
    s2 = lumina.Scene(sc.camera, sc.sun, tris, sc.mat_albedo, sc.mat_emissive, sc.points, textures=sc.textures)
    r = lumina.Renderer(0)
    r.set_scene_bvh(s2, nodes)
    r.set_bvh_width(width)
    loaded, missing = r.load_textures(str(root))
    assert (loaded, missing) == (len(sc.textures) - 1, 1)
    O.ref_set_textures([str(root / t) for t in sc.textures])
    return r, nodes, tris


@pytest.mark.parametrize("width", [2, 4])
def test_textured_render_vs_reference_gpu(textured, width):
    if not O.ref_available():
        pytest.skip("reference oracle not built")
    sc, root = textured
    r, nodes, tris = _setup(sc, root, width)
    try:
        ours = r.render(spp=8, bounces=2)
        ref_acc, ref_rgb, _ = O.ref_render_gpu(sc, nodes, tris, 8, 2)
    finally:
        r.close()
        O.ref_set_textures([])
    close = np.abs(ours["accum"] - ref_acc) <= REL * np.maximum(np.abs(ours["accum"]), np.abs(ref_acc)) + ABS
    assert float(close.all(axis=2).mean()) >= 0.999
    assert float((ours["rgb"] == ref_rgb).all(axis=2).mean()) >= 0.999
    # the textures do change the image
    with lumina.Renderer(0) as plain:
        s2 = lumina.Scene(sc.camera, sc.sun, tris, sc.mat_albedo, sc.mat_emissive, sc.points)
        plain.set_scene_bvh(s2, nodes)
        assert not np.array_equal(plain.render(spp=8, bounces=2)["rgb"], ours["rgb"])


def test_textured_gbuffer_vs_reference_gpu(textured):
    if not O.ref_available():
        pytest.skip("reference oracle not built")
    sc, root = textured
    r, nodes, tris = _setup(sc, root, 4)
    try:
        ours = r.gbuffer()
        ref = O.ref_gbuffer_gpu(sc, nodes, tris)
    finally:
        r.close()
        O.ref_set_textures([])
    for a, b in zip(ours, ref):
        assert float((a == b).all(axis=2).mean()) >= 0.999


def test_cli_textures(textured):
    sc, root = textured
    out = root / "t.png"  # as in the reference, a single render does not create directories
    scene = root / "scenes" / "scene.json"
    r = subprocess.run([str(_ffi.CLI_PATH), str(scene), str(out), "--spp", "2", "--bounces", "1"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    n = len(sc.textures)
    assert f"textures: {n - 1} loaded, 1 missing (of {n} materials)" in r.stdout
    assert f"texture not found: {root}/tex/missing.png" in r.stderr
    from PIL import Image
    got = np.asarray(Image.open(out).convert("RGB"))
    with lumina.Renderer(0) as rr:
        loaded = lumina.Scene.load_json(scene)
        rr.set_scene(loaded)
        rr.load_textures(str(root))
        want = rr.render(spp=2, bounces=1)["rgb"]
    assert np.array_equal(got, want)
