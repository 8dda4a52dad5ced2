"""Field-slice PNG output (gdiamond_b200/snapshot.py) against the reference's save_field_png
(gDiamond/utils.h:210-255), CPU only.

* the colour map against the PNG the reference wrote for a seeded slice (committed fixture,
  tests/golden/ref_png_37x23.npz) and, when oracle/_ref is built, against the reference run
  here on another slice;
* the PNG encoder round-trips through an independent decoder (every PNG row filter handled,
  since stb_image_write picks one per row).
"""
import os
import struct
import zlib

import numpy as np
import pytest

import oracle
from gdiamond_b200 import snapshot as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def decode_png(data):
    """uint8 [h][w][3] pixels of an 8-bit RGB, non-interlaced PNG."""
    data = bytes(data)
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", None
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        assert zlib.crc32(tag + body) & 0xFFFFFFFF == struct.unpack(">I", data[pos + 8 + n:
                                                                            pos + 12 + n])[0]
        if tag == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
            assert (depth, ctype, interlace) == (8, 2, 0)
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    stride, bpp = w * 3, 3
    out = np.zeros((h, stride), np.uint8)
    prev = [0] * stride
    for y in range(h):
        ft = raw[y * (stride + 1)]
        line = raw[y * (stride + 1) + 1:(y + 1) * (stride + 1)]
        cur = [0] * stride
        for x in range(stride):
            a = cur[x - bpp] if x >= bpp else 0
            b = prev[x]
            c = prev[x - bpp] if x >= bpp else 0
            if ft == 0:
                pred = 0
            elif ft == 1:
                pred = a
            elif ft == 2:
                pred = b
            elif ft == 3:
                pred = (a + b) // 2
            elif ft == 4:
                p = a + b - c
                pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                pred = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            else:
                raise ValueError(f"filter {ft}")
            cur[x] = (line[x] + pred) & 255
        out[y] = cur
        prev = cur
    return out.reshape(h, w, 3)


def test_colour_map_matches_reference_golden_png():
    d = np.load(os.path.join(GOLDEN, "ref_png_37x23.npz"))
    want = decode_png(d["png"])
    got = P.diverging_rgb(d["u"], d["vmax"])
    assert want.shape == got.shape == (23, 37, 3)
    assert np.array_equal(got, want)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_colour_map_matches_reference_run_here(tmp_path):
    rng = np.random.default_rng(3)
    u = (rng.standard_normal((41, 64)) * np.float32(0.7)).astype(np.float32)
    u[5, 5], u[6, 6] = np.float32(-0.0), np.float32(0.7)
    path = str(tmp_path / "ref.png")
    oracle.ref_save_field_png(u, path, 0.7)
    assert np.array_equal(P.diverging_rgb(u, 0.7), decode_png(open(path, "rb").read()))


def test_png_encoder_round_trip(tmp_path):
    rng = np.random.default_rng(9)
    rgb = rng.integers(0, 256, (17, 29, 3), dtype=np.uint8)
    assert np.array_equal(decode_png(P.encode_png(rgb)), rgb)
    with pytest.raises(ValueError):
        P.encode_png(np.zeros((4, 4, 4), np.uint8))
