"""Image metrics as the reference's tools compute them.

* psnr: tools/diff.py:25-29 -- FP64 MSE over 8-bit images, 20*log10(255/sqrt(MSE)).
* mad:  tools/diff.py:103 -- mean |a - b| over all channels.
* ssim: skimage.metrics.structural_similarity as tools/diff.py:100 calls it
  (channel_axis=2, data_range=255), restated from Wang et al. 2004 with
  skimage's defaults: 7x7 uniform window (reflect padding), sample
  covariance (N/(N-1)), K1=0.01, K2=0.03, mean over the window-valid
  interior, then over channels.  (skimage itself is not a dependency.)
"""
from __future__ import annotations

import numpy as np


def psnr(a: np.ndarray, b: np.ndarray, data_range: float = 255.0) -> float:
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    if mse == 0:
        return float("inf")
    return float(20.0 * np.log10(data_range / np.sqrt(mse)))


def mad(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.mean(np.abs(a.astype(np.int16) - b.astype(np.int16))))


def _ssim_channel(x: np.ndarray, y: np.ndarray, data_range: float, win: int = 7) -> float:
    from scipy.ndimage import uniform_filter

    K1, K2 = 0.01, 0.03
    np_ = win * win
    cov_norm = np_ / (np_ - 1.0)
    ux = uniform_filter(x, size=win)
    uy = uniform_filter(y, size=win)
    uxx = uniform_filter(x * x, size=win)
    uyy = uniform_filter(y * y, size=win)
    uxy = uniform_filter(x * y, size=win)
    vx = cov_norm * (uxx - ux * ux)
    vy = cov_norm * (uyy - uy * uy)
    vxy = cov_norm * (uxy - ux * uy)
    C1 = (K1 * data_range) ** 2
    C2 = (K2 * data_range) ** 2
    A1, A2 = 2 * ux * uy + C1, 2 * vxy + C2
    B1, B2 = ux * ux + uy * uy + C1, vx + vy + C2
    S = (A1 * A2) / (B1 * B2)
    pad = (win - 1) // 2
    return float(S[pad:-pad, pad:-pad].mean())


def ssim(a: np.ndarray, b: np.ndarray, data_range: float = 255.0) -> float:
    """(H, W, C) or (H, W) images."""
    x = a.astype(np.float64)
    y = b.astype(np.float64)
    if x.ndim == 2:
        return _ssim_channel(x, y, data_range)
    return float(np.mean([_ssim_channel(x[..., c], y[..., c], data_range) for c in range(x.shape[2])]))


def tonemap_u8(linear: np.ndarray) -> np.ndarray:
    """The renderer's display encode (pathtracer.cu:413-429): sqrt(clamp(v, 0, 1)) * 255, truncated."""
    v = np.sqrt(np.clip(linear.astype(np.float32), 0.0, 1.0)) * np.float32(255.0)
    return v.astype(np.uint8)
