"""diff report: PSNR / SSIM / MAD and an absolute-difference heatmap.

Drop-in for the reference's tools/diff.py (tools/diff.py:85-119): same
command line (`diff.py engine.png ref.png [--out report.html]`), same
printed line (`PSNR x dB | SSIM y | MAD z`), same report contents (metrics
table, the two images and a x4 heatmap through the same hand-made
viridis-like ramp, tools/diff.py:32-46), without the scikit-image
dependency (lumina.metrics.ssim restates its SSIM).

    python -m lumina.diff engine.png ref.png --out report.html
"""
from __future__ import annotations

import argparse
import base64
import io
import pathlib
import sys

import numpy as np

from . import metrics


def load_rgb(path):
    from PIL import Image
    img = Image.open(path).convert("RGB")
    return np.asarray(img, dtype=np.uint8), img.size


def match_size(a, target_wh):
    from PIL import Image
    if (a.shape[1], a.shape[0]) == target_wh:
        return a
    return np.asarray(Image.fromarray(a).resize(target_wh, Image.BILINEAR), dtype=np.uint8)


def ramp_lut() -> np.ndarray:
    """256-entry colour ramp: quadratic fits per channel, as tools/diff.py:32-38."""
    x = np.linspace(0.0, 1.0, 256)
    r = np.clip(-0.2 + 2.4 * x - 1.3 * x ** 2, 0, 1)
    g = np.clip(0.1 + 0.8 * x + 0.1 * x ** 2, 0, 1)
    b = np.clip(0.4 + 0.8 * x - 1.1 * x ** 2, 0, 1)
    return (np.stack([r, g, b], axis=1) * 255).astype(np.uint8)


def heatmap(a, b, gain=4.0):
    d = np.mean(np.abs(a.astype(np.int16) - b.astype(np.int16)), axis=2)
    d = np.clip(d * gain, 0, 255).astype(np.uint8)
    return ramp_lut()[d]


def _b64(arr):
    from PIL import Image
    buf = io.BytesIO()
    Image.fromarray(arr).save(buf, format="PNG")
    return base64.b64encode(buf.getvalue()).decode("ascii")


_PAGE = """<!doctype html>
<html><head><meta charset="utf-8"><title>Diff Report</title>
<style>body{{font-family:sans-serif;margin:1.5em;color:#eee;background:#222}}
td,th{{padding:.3em 1em;border-bottom:1px solid #555;text-align:left}}th{{color:#aaa;font-weight:normal}}
.grid{{display:grid;grid-template-columns:repeat(3,1fr);gap:1em}}.grid img{{width:100%;border:1px solid #444}}
figcaption{{color:#aaa;font-size:.9em}}</style></head><body>
<h1>LuminaGI vs CUDA Reference</h1>
<table><tr><th>Resolution</th><td>{w}x{h}</td></tr><tr><th>PSNR</th><td>{psnr:.2f} dB</td></tr>
<tr><th>SSIM</th><td>{ssim:.4f}</td></tr><tr><th>Mean abs diff (per channel)</th><td>{mad:.2f} / 255</td></tr>
<tr><th>Engine</th><td>{a}</td></tr><tr><th>Reference</th><td>{b}</td></tr></table>
<div class="grid"><figure><img src="data:image/png;base64,{ia}"><figcaption>Engine (LuminaGI)</figcaption></figure>
<figure><img src="data:image/png;base64,{ib}"><figcaption>Reference (CUDA)</figcaption></figure>
<figure><img src="data:image/png;base64,{ih}"><figcaption>Abs diff &times; 4</figcaption></figure></div>
</body></html>
"""


def report(engine_path, ref_path, out_path):
    engine, eng_size = load_rgb(engine_path)
    ref, ref_size = load_rgb(ref_path)
    if eng_size != ref_size:
        print(f"resizing engine {eng_size} -> {ref_size}", file=sys.stderr)
        engine = match_size(engine, ref_size)
    p, s, m = metrics.psnr(engine, ref), metrics.ssim(engine, ref), metrics.mad(engine, ref)
    heat = heatmap(engine, ref)
    from PIL import Image
    Image.fromarray(heat).save(pathlib.Path(out_path).with_suffix(".heatmap.png"))
    html = _PAGE.format(w=ref_size[0], h=ref_size[1], psnr=p, ssim=s, mad=m,
                        a=pathlib.Path(engine_path).resolve().as_posix(), b=pathlib.Path(ref_path).resolve().as_posix(),
                        ia=_b64(engine), ib=_b64(ref), ih=_b64(heat))
    pathlib.Path(out_path).write_text(html, encoding="utf-8")
    return p, s, m


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("engine", help="LuminaGI screenshot PNG")
    ap.add_argument("ref", help="CUDA reference PNG")
    ap.add_argument("--out", default="diff_report.html")
    a = ap.parse_args(argv)
    p, s, m = report(a.engine, a.ref, a.out)
    print(f"PSNR {p:.2f} dB | SSIM {s:.4f} | MAD {m:.2f}")
    print(f"wrote {a.out}")


if __name__ == "__main__":
    main()
