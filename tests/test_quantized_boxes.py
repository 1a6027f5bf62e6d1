"""The grid rule of the quantized 4-wide traversal records, restated in numpy
(luminagi-cudaref_b200/csrc/trace.cu, quantize_axis), and the property the
traversal relies on: every child's quantized planes lie at least one grid step
outside its exact box, and every plane fits in one byte.  Random, flat,
far-from-origin and tiny boxes."""
import math

import numpy as np
import pytest


def quantize_axis(lo, hi):
    """lo, hi: float32 arrays of the present children's planes on one axis."""
    pl, ph = float(np.min(lo)), float(np.max(hi))
    ext = ph - pl
    m = max(abs(pl), abs(ph))
    E = -126
    if ext > 0.0:
        E = max(E, math.ceil(math.log2(ext / 252.0)))
    if m > 0.0:
        E = max(E, math.frexp(m)[1] - 1 - 22)  # ilogb(m) - 22
    E = min(E, 127)
    step = math.ldexp(1.0, E)
    o = np.float32(pl - step)
    if float(o) > pl - step:  # round toward -inf
        o = np.nextafter(o, np.float32(-np.inf))
    origin = float(o)
    ql = [min(255, max(0, math.floor((float(a) - origin) / step) - 1)) for a in lo]
    qh = [min(255, max(0, math.ceil((float(b) - origin) / step) + 1)) for b in hi]
    return origin, step, ql, qh


def check(lo, hi):
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    origin, step, ql, qh = quantize_axis(lo, hi)
    assert float(np.float32(step)) == step  # a normal power of two
    for k in range(len(lo)):
        assert 0 <= ql[k] <= 255 and 0 <= qh[k] <= 255
        assert origin + ql[k] * step <= float(lo[k]) - step
        assert origin + qh[k] * step >= float(hi[k]) + step


@pytest.mark.parametrize("scale,offset", [(1.0, 0.0), (1e-3, 20.0), (40.0, -20.0), (1e-6, 1e4), (1e3, 0.0)])
def test_random_children(scale, offset):
    rng = np.random.default_rng(7)
    for _ in range(2000):
        k = int(rng.integers(1, 5))
        a = (rng.random((k, 2)) * scale + offset).astype(np.float32)
        check(a.min(axis=1), a.max(axis=1))


def test_flat_and_degenerate_axes():
    check([5.0], [5.0])  # a flat box (axis-aligned quad)
    check([0.0, 0.0], [0.0, 0.0])
    check([-0.0], [0.0])
    check([19.999998, 20.0], [20.0, 20.000002])  # extent of a few ulps
    check([np.float32(3e38)], [np.float32(3e38)])
    check([-1e-30], [1e-30])
