"""What the trained network gains over the method without it.

A small seeded engine-style scene (64x64 grids, 3-subdivision spheres) is
rendered on the device at 10 orbit poses as (8-spp, 256-spp) pairs; the UNet
is trained on 8 of them with this library's own forward, backward and Adam
kernels (L1, best-validation parameters kept, as ml/train.py:128-225 does);
the 2 held-out poses are judged against 1024-spp renders accumulated in FP64.
PSNR is the reference's (tools/diff.py:25-29) on the 8-bit sqrt-tonemapped
images.

Bars: the trained denoiser's held-out PSNR beats the plain 8-spp render by
at least 3 dB, and beats the same network before training (He-initialised
weights: the output is the noisy input plus a random residual) by at least
3 dB.  Training is not bit-reproducible (FP32 atomics in the weight
gradients), so the bars leave room below the gains measured on B200."""
import numpy as np
import pytest

import lumina
from lumina import surrogate as S
from lumina.scene import ENGINE_CENTER, orbit_poses

pytestmark = pytest.mark.gpu

MARGIN_DB = 3.0


def test_trained_denoiser_gains_over_the_plain_render(small_engine_scene):
    torch = pytest.importorskip("torch")
    sc = lumina.engine_scene(seed=7, width=256, height=128, grid_n=64, sphere_subdiv=3)
    r = lumina.Renderer(0)
    r.set_scene(sc)
    cams = [sc.camera.look_at(p, t) for p, t in orbit_poses(10, seed=11, center=ENGINE_CENTER)]
    noisy, clean = S.make_dataset(r, cams, 8, 256, 2)
    val_idx, train_idx = [3, 7], [i for i in range(10) if i not in (3, 7)]
    frames = S.eval_frames(r, [cams[i] for i in val_idx], 8, 256, 1024, 2)

    net = lumina.UNet()
    init = S.he_init(42)
    net.set_params(init)
    before, _ = S.evaluate(net, frames)
    # 60 epochs x 8 poses x 6 crops of 64 px, batches of 8: 360 Adam steps
    best, best_val, hist = S.train(net, noisy, clean, train_idx, val_idx, epochs=60, batch=8, crop=64, lr=3e-4,
                                   crops_per_image=6, seed=42, log=None)
    net.set_params(best)
    after, _ = S.evaluate(net, frames)
    net.close()
    r.close()
    print(f"held-out PSNR vs FP64 judge: 8 spp {after['noisy_psnr']:.2f} dB, untrained net "
          f"{before['denoised_psnr']:.2f} dB, trained net {after['denoised_psnr']:.2f} dB, 256 spp "
          f"{after['clean_psnr']:.2f} dB; train L1 {hist[0][1]:.4f} -> {hist[-1][1]:.4f}, best val {best_val:.4f}")
    assert hist[-1][1] < hist[0][1]
    assert after["denoised_psnr"] >= after["noisy_psnr"] + MARGIN_DB
    assert after["denoised_psnr"] >= before["denoised_psnr"] + MARGIN_DB
    assert after["denoised_ssim"] > after["noisy_ssim"]
