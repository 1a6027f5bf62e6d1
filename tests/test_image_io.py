"""PNG decoding (lg_image_load), the texture loader behind diffuse_tex.

Every colour type, bit depth, filter and Adam7 interlacing, encoded by
tests/pngenc.py and checked (a) against the conversion rules of stb_image's
4-channel load and (b) against the reference's own stbi_load (compiled into
the reference oracle) on the same files."""
import itertools

import numpy as np
import pytest

import lumina
import oracle as O
import pngenc

CASES = [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (2, 8), (2, 16), (3, 1), (3, 2), (3, 4), (3, 8), (4, 8), (4, 16),
         (6, 8), (6, 16)]
SIZES = [(1, 1), (7, 13), (16, 9), (33, 5)]


def make_case(ctype, depth, h, w, seed, with_trns):
    rng = np.random.default_rng(seed)
    C = pngenc.CHANNELS[ctype]
    palette = trns = None
    if ctype == 3:
        n_pal = min(1 << depth, 200)
        samples = rng.integers(0, n_pal, (h, w, 1))
        palette = rng.integers(0, 256, (n_pal, 3))
        if with_trns:
            trns = list(rng.integers(0, 256, max(1, n_pal // 2)))
    else:
        samples = rng.integers(0, 1 << depth, (h, w, C))
        if with_trns and ctype == 0:
            k = int(samples[0, 0, 0])
            trns = [k >> 8, k & 255]
        if with_trns and ctype == 2:
            trns = sum(([int(v) >> 8, int(v) & 255] for v in samples[0, 0]), [])
    return samples, palette, trns


@pytest.mark.parametrize("ctype,depth", CASES)
@pytest.mark.parametrize("interlace", [False, True])
def test_decode_all_forms(tmp_path, ctype, depth, interlace):
    for (h, w), with_trns in itertools.product(SIZES, [False, True]):
        if with_trns and ctype in (4, 6):
            continue
        seed = hash((ctype, depth, interlace, h, w, with_trns)) & 0xFFFF
        samples, palette, trns = make_case(ctype, depth, h, w, seed, with_trns)
        data = pngenc.encode(samples, ctype, depth, interlace, palette, trns, seed=seed, idat_split=37)
        p = tmp_path / f"c{ctype}_d{depth}_i{int(interlace)}_{h}x{w}_{int(with_trns)}.png"
        p.write_bytes(data)
        got = lumina.load_image(p)
        want = pngenc.expected_rgba(samples, ctype, depth, palette, trns)
        assert got.shape == (h, w, 4)
        assert np.array_equal(got, want), p.name
        if O.ref_available():
            ref = O.ref_image_load(p)
            assert ref is not None and np.array_equal(got, ref), p.name


def test_decode_pil_written(tmp_path):
    """Files written by another encoder (Pillow), including its palette/optimise paths."""
    Image = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(3)
    rgb = rng.integers(0, 256, (37, 21, 3), dtype=np.uint8)
    for mode in ("RGB", "RGBA", "L", "LA", "P", "1"):
        im = Image.fromarray(rgb).convert(mode)
        p = tmp_path / f"pil_{mode}.png"
        im.save(p, optimize=True)
        got = lumina.load_image(p)
        want = np.asarray(im.convert("RGBA"))
        assert np.array_equal(got, want), mode
        if O.ref_available():
            assert np.array_equal(got, O.ref_image_load(p)), mode


def test_errors(tmp_path):
    with pytest.raises(FileNotFoundError):
        lumina.load_image(tmp_path / "missing.png")
    bad = tmp_path / "not.png"
    bad.write_bytes(b"GIF89a....")
    with pytest.raises(OSError):
        lumina.load_image(bad)
    good = pngenc.encode(np.zeros((4, 4, 3), np.int64), 2, 8)
    trunc = tmp_path / "trunc.png"
    trunc.write_bytes(good[:40])
    with pytest.raises(OSError):
        lumina.load_image(trunc)
    # a bad CRC is accepted, as stb_image accepts it
    crc = bytearray(good)
    crc[29] ^= 0xFF  # IHDR CRC byte
    p = tmp_path / "crc.png"
    p.write_bytes(bytes(crc))
    assert lumina.load_image(p).shape == (4, 4, 4)
