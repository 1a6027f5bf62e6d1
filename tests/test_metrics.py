"""PSNR / MAD / SSIM as the reference's tools compute them.

Known answers: the reference's published numbers for its shipped renders
(README.md:103-105, docs/denoiser.md:30-32) against ml/eval/gt_1024.png --
PSNR 34.52 / 42.04 / 49.57 dB, MAD 3.25 / 1.39 / 0.51, SSIM 0.815 / 0.964 /
0.991 (three decimals) -- checked when the reference checkout is present,
plus closed-form cases that always run."""
import os
import pathlib

import numpy as np
import pytest

from lumina import metrics as M

# The reference checkout (same variable as oracle/Makefile); its shipped renders sit under ml/eval.
EVAL = pathlib.Path(os.environ.get("REF", "/root/reference")) / "ml" / "eval"
KAT = [("noisy_8", 34.52, 3.25, 0.815), ("denoised", 42.04, 1.39, 0.964), ("clean_256", 49.57, 0.51, 0.991)]


@pytest.mark.skipif(not (EVAL / "gt_1024.png").exists(), reason="reference renders not present")
@pytest.mark.parametrize("name,psnr,mad,ssim", KAT)
def test_published_metrics_reproduce(name, psnr, mad, ssim):
    from PIL import Image
    gt = np.asarray(Image.open(EVAL / "gt_1024.png").convert("RGB"))
    a = np.asarray(Image.open(EVAL / f"{name}.png").convert("RGB"))
    assert round(M.psnr(a, gt), 2) == psnr
    assert round(M.mad(a, gt), 2) == mad
    assert abs(M.ssim(a, gt) - ssim) < 1e-3


def test_closed_forms():
    rng = np.random.default_rng(1)
    a = rng.integers(0, 200, (40, 50, 3), dtype=np.uint8)
    assert M.psnr(a, a) == float("inf") and M.ssim(a, a) == pytest.approx(1.0)
    b = a + np.uint8(5)
    assert M.psnr(a, b) == pytest.approx(20 * np.log10(255 / 5))
    assert M.mad(a, b) == pytest.approx(5.0)
    assert M.ssim(a, 255 - a) < 0.0


def test_tonemap_matches_oracle():
    import oracle as O
    acc = np.random.default_rng(2).uniform(-0.5, 3.0, (8, 9, 3)).astype(np.float32)
    assert np.array_equal(M.tonemap_u8(acc), O.oracle_tonemap(acc, 1))


def test_diff_report_cli(tmp_path):
    import subprocess
    import sys
    from PIL import Image
    rng = np.random.default_rng(4)
    a = rng.integers(0, 256, (24, 40, 3), dtype=np.uint8)
    b = np.clip(a.astype(int) + rng.integers(-3, 4, a.shape), 0, 255).astype(np.uint8)
    pa, pb = tmp_path / "a.png", tmp_path / "b.png"
    Image.fromarray(a).save(pa)
    Image.fromarray(b).save(pb)
    out = tmp_path / "r.html"
    pkg = pathlib.Path(__file__).resolve().parent.parent / "luminagi-cudaref_b200"
    r = subprocess.run([sys.executable, "-m", "lumina.diff", str(pa), str(pb), "--out", str(out)], cwd=pkg,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert f"PSNR {M.psnr(a, b):.2f} dB | SSIM {M.ssim(a, b):.4f} | MAD {M.mad(a, b):.2f}" in r.stdout
    assert out.exists() and out.with_suffix(".heatmap.png").exists()
    heat = np.asarray(Image.open(out.with_suffix(".heatmap.png")))
    assert heat.shape == (24, 40, 3)
