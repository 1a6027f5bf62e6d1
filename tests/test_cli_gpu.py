"""The cuda_ref CLI (drop-in for the reference's src/main.cpp) and the
denoiser's 8-bit I/O contract (tools/denoise.py), on the GPU."""
import subprocess

import numpy as np
import pytest

import lumina
from lumina import _ffi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_box(tmp_path_factory):
    sc = lumina.box_scene(3, width=96, height=48, sphere_subdiv=2)
    d = tmp_path_factory.mktemp("cli")
    p = d / "scene.json"
    sc.save_json(p)
    return sc, p, d


def _png(p):
    from PIL import Image
    return np.asarray(Image.open(p).convert("RGB"))


def test_single_render_matches_library(small_box):
    sc, p, d = small_box
    out = d / "out.png"
    r = subprocess.run([str(_ffi.CLI_PATH), str(p), str(out), "--spp", "4", "--bounces", "1", "--hdr",
                        str(d / "out.hdr")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for needle in ("[scene] loaded", "bvh:", "kernel:", "render:", f"wrote {out}"):
        assert needle in r.stdout
    assert (d / "out.hdr").exists()
    with lumina.Renderer(0) as rr:
        rr.set_scene(sc)
        ref = rr.render(spp=4, bounces=1)["rgb"]
    assert np.array_equal(_png(out), ref)


def test_camera_override(small_box):
    sc, p, d = small_box
    out = d / "cam.png"
    r = subprocess.run([str(_ffi.CLI_PATH), str(p), "-o", str(out), "--spp", "2", "--bounces", "0", "--cam-pos",
                        "-3", "2", "2.5", "--cam-target", "0", "0", "1"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "camera override: pos (-3.00,2.00,2.50) -> target (0.00,0.00,1.00)" in r.stdout
    cam = sc.camera.look_at([-3, 2, 2.5], [0, 0, 1])
    with lumina.Renderer(0) as rr:
        rr.set_scene(sc)
        ref = rr.render(camera=cam, spp=2, bounces=0)["rgb"]
    assert np.array_equal(_png(out), ref)


def test_batch_mode(small_box):
    sc, p, d = small_box
    jobs = d / "batch.txt"
    a, b = d / "j" / "a.png", d / "j" / "b.png"
    jobs.write_text(f"# out_png spp bounces  camx camy camz  tgtx tgty tgtz\n"
                    f"{a} 8 2 -3.0 -1.0 2.0 0 0 1  # first\n"
                    f"this line is malformed\n"
                    f"{b} 3 0 2.5 2.5 3.0 0 0 0.5\n")
    r = subprocess.run([str(_ffi.CLI_PATH), str(p), "--batch", str(jobs)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "batch: 2 jobs" in r.stdout and "[1/2]" in r.stdout and "[2/2]" in r.stdout
    with lumina.Renderer(0) as rr:
        rr.set_scene(sc)
        ra = rr.render(camera=sc.camera.look_at([-3, -1, 2], [0, 0, 1]), spp=8, bounces=2)["rgb"]
        rb = rr.render(camera=sc.camera.look_at([2.5, 2.5, 3], [0, 0, 0.5]), spp=3, bounces=0)["rgb"]
    assert np.array_equal(_png(a), ra) and np.array_equal(_png(b), rb)


def test_denoise_rgb8_contract():
    """tools/denoise.py: u8/255 -> replicate-pad to x8 -> net -> crop -> clip*255+0.5."""
    torch = pytest.importorskip("torch")
    import unet_ref
    flat = unet_ref.make_params(9)
    net = lumina.UNet()
    net.set_params(flat)
    img = np.random.default_rng(1).integers(0, 256, (21, 30, 3), dtype=np.uint8)
    got = net.denoise_rgb8(img)
    assert got.shape == img.shape and got.dtype == np.uint8
    m = unet_ref.load_flat(unet_ref.UNetRef().eval(), flat)
    x = torch.from_numpy(img.astype(np.float32).transpose(2, 0, 1)[None] / 255.0)
    x = torch.nn.functional.pad(x, (0, 2, 0, 3), mode="replicate")
    with torch.no_grad():
        # the library's inference pass folds u3a/u2a/u1a's upsampled inputs (lg_unet_set_fold_upsampling)
        y = unet_ref.forward_bf16(m, x, fold=("u3", "u2", "u1"))[0, :, :21, :30].numpy().transpose(1, 2, 0)
    ref = (np.clip(y, 0, 1) * 255.0 + 0.5).astype(np.uint8)
    # BF16 summation-order noise is ~0.4 of an 8-bit step (see test_unet_forward_matches_torch).
    diff = np.abs(got.astype(int) - ref.astype(int))
    assert diff.max() <= 6 and np.mean(diff <= 1) > 0.95


def test_gbuffer_outputs(small_box):
    """--gbuffer writes <stem>.albedo/.normal/.worldpos.png beside the colour image (main.cpp:177-184)."""
    sc, p, d = small_box
    out = d / "g" / "frame.png"
    r = subprocess.run([str(_ffi.CLI_PATH), str(p), str(out), "--spp", "1", "--bounces", "0", "--gbuffer"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    with lumina.Renderer(0) as rr:
        rr.set_scene(sc)
        ref = rr.gbuffer()
    for name, img in zip(("albedo", "normal", "worldpos"), ref):
        f = d / "g" / f"frame.{name}.png"
        assert f.exists()
        assert np.array_equal(_png(f), img)


@pytest.mark.parametrize("in_ch", [3, 12])
def test_denoise_cli(tmp_path, in_ch):
    """python -m lumina.denoise (tools/denoise.py drop-in) on a reference-format checkpoint."""
    import sys
    from lumina import surrogate
    params = surrogate.he_init(5, in_ch)
    ck = tmp_path / "ck.pt"
    surrogate.save_checkpoint(params, str(ck), in_ch)
    rng = np.random.default_rng(in_ch)
    imgs = [rng.integers(0, 256, (21, 30, 3), dtype=np.uint8) for _ in range(4)]
    names = ["frame.png", "frame.albedo.png", "frame.normal.png", "frame.worldpos.png"]
    for n, im in zip(names, imgs):
        lumina.lib().lg_write_png(str(tmp_path / n).encode(), 30, 21, np.ascontiguousarray(im).ctypes.data)
    out = tmp_path / "den.png"
    r = subprocess.run([sys.executable, "-m", "lumina.denoise", str(ck), str(tmp_path / "frame.png"), str(out)],
                       capture_output=True, text=True, cwd=str(_ffi.PKG_DIR))
    assert r.returncode == 0, r.stderr
    assert "inference:" in r.stdout and "(30x21, base=32)" in r.stdout
    net = lumina.UNet(in_ch=in_ch)
    net.set_params(params)
    want = net.denoise_rgb8(*imgs[:1 if in_ch == 3 else 4])
    assert np.array_equal(_png(out), want)
