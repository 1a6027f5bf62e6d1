"""A small PNG encoder for tests: any colour type, bit depth, Adam7
interlacing and per-row filter choice, so the decoder is exercised on every
form the PNG specification allows.  Written from the specification."""
from __future__ import annotations

import struct
import zlib

import numpy as np

CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}
ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]


def _chunk(t: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + t + data + struct.pack(">I", zlib.crc32(t + data) & 0xFFFFFFFF)


def _pack_row(samples: np.ndarray, depth: int) -> bytes:
    """samples: (n,) unsigned ints for one row (channels interleaved)."""
    if depth == 8:
        return samples.astype(np.uint8).tobytes()
    if depth == 16:
        return samples.astype(">u2").tobytes()
    per = 8 // depth
    n = len(samples)
    out = bytearray((n * depth + 7) // 8)
    for i, v in enumerate(samples):
        out[i // per] |= (int(v) & ((1 << depth) - 1)) << (8 - depth * (i % per + 1))
    return bytes(out)


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    if pa <= pb and pa <= pc:
        return a
    return b if pb <= pc else c


def _filter(rows, bpp, rng):
    out = bytearray()
    prev = bytes(len(rows[0])) if rows else b""
    for r in rows:
        f = int(rng.integers(0, 5))
        line = bytearray(len(r))
        for i in range(len(r)):
            a = r[i - bpp] if i >= bpp else 0
            b = prev[i]
            c = prev[i - bpp] if i >= bpp else 0
            pred = [0, a, b, (a + b) >> 1, _paeth(a, b, c)][f]
            line[i] = (r[i] - pred) & 0xFF
        out.append(f)
        out += line
        prev = r
    return bytes(out)


def encode(samples: np.ndarray, ctype: int, depth: int, interlace: bool = False, palette=None, trns=None,
           seed: int = 0, idat_split: int = 0) -> bytes:
    """samples: (H, W, channels) unsigned ints at `depth` bits (palette indices for ctype 3)."""
    H, W, C = samples.shape
    assert C == CHANNELS[ctype]
    rng = np.random.default_rng(seed)
    bits = C * depth
    bpp = max(1, bits // 8)
    raw = bytearray()
    passes = ADAM7 if interlace else [(0, 0, 1, 1)]
    for x0, y0, dx, dy in passes:
        sub = samples[y0::dy, x0::dx]
        if sub.shape[0] == 0 or sub.shape[1] == 0:
            continue
        rows = [_pack_row(sub[y].reshape(-1), depth) for y in range(sub.shape[0])]
        raw += _filter(rows, bpp, rng)
    z = zlib.compress(bytes(raw), 9)
    out = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, depth, ctype, 0, 0, int(interlace)))
    if palette is not None:
        out += _chunk(b"PLTE", np.asarray(palette, np.uint8).reshape(-1).tobytes())
    if trns is not None:
        out += _chunk(b"tRNS", bytes(trns))
    if idat_split:
        for i in range(0, len(z), idat_split):
            out += _chunk(b"IDAT", z[i:i + idat_split])
    else:
        out += _chunk(b"IDAT", z)
    return out + _chunk(b"IEND", b"")


def expected_rgba(samples, ctype, depth, palette=None, trns=None) -> np.ndarray:
    """8-bit RGBA as stb_image's 4-channel load produces it."""
    H, W, _ = samples.shape
    s = samples.astype(np.int64)

    def to8(v):
        if depth == 16:
            return v >> 8
        return v * {1: 0xFF, 2: 0x55, 4: 0x11, 8: 1}[depth]

    out = np.full((H, W, 4), 255, np.int64)
    if ctype == 0:
        out[..., :3] = to8(s[..., :1])
        if trns is not None:
            key = trns[0] << 8 | trns[1]
            out[..., 3][s[..., 0] == key] = 0
    elif ctype == 2:
        out[..., :3] = to8(s)
        if trns is not None:
            key = [trns[2 * k] << 8 | trns[2 * k + 1] for k in range(3)]
            out[..., 3][(s[..., 0] == key[0]) & (s[..., 1] == key[1]) & (s[..., 2] == key[2])] = 0
    elif ctype == 3:
        pal = np.asarray(palette, np.int64).reshape(-1, 3)
        out[..., :3] = pal[s[..., 0]]
        if trns is not None:
            a = np.full(len(pal), 255, np.int64)
            a[:len(trns)] = list(trns)
            out[..., 3] = a[s[..., 0]]
    elif ctype == 4:
        out[..., :3] = to8(s[..., :1])
        out[..., 3] = to8(s[..., 1])
    elif ctype == 6:
        out[...] = to8(s)
    return out.astype(np.uint8)
